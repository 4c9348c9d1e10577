// Wavefront MIS path tracer on the GPU: the device side of the su_* render entry points.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "material.cuh"

namespace spb::render {

// A density grid (one-channel 3-D image, su_create_image), x fastest then y then z.
struct Density_grid {
    uint32_t     dims[3] = {0, 0, 0};
    float const* density = nullptr;  // dims[0] * dims[1] * dims[2] values, read during set_scene
};

// One prop filled with a heterogeneous medium (Grid material, volumetric_grid.cpp): the grid it
// samples and the map from world space to the grid's texture space [0, 1]^3 (the prop's
// world-to-object transformation followed by its mesh bounds, tracking.inl:12-29).
struct Grid_medium {
    uint32_t grid           = 0;      // index into Scene_desc::grids
    bool     nearest        = false;  // Nearest_3D filter instead of Linear_3D
    bool     repeat         = false;  // Address_mode_repeat instead of clamp
    float    world_to_uvw[12] = {};   // rows: uvw_k = dot(row_k.xyz, p) + row_k.w
    // An emitting grid's temperature (Grid_emission::set_temperature_map): 1 + index into
    // Scene_desc::grids of a grid of the density's dimensions, 0 for none; and the material's
    // emission times the black-body colour at 2000 + 200 k kelvin for k = 0..15 (RGB triples),
    // looked up by temperature over [0, 1.2] (volumetric_grid.cpp:140-160).
    uint32_t temperature    = 0;
    float    blackbody[48]  = {};
    // A two-channel density's second channel, which scales the emission (Grid_emission,
    // volumetric_grid.cpp:80-127): 1 + index into Scene_desc::grids, 0 for none.
    uint32_t emission_scale = 0;
    // A colour grid (Grid_color, volumetric_grid.cpp:336-395): `grid` is its alpha, these its
    // red, green and blue (1 + index into Scene_desc::grids each, 0 for a density grid); the
    // coefficients are alpha x attenuation(rgb, rgb, color_distance, anisotropy).
    uint32_t color[3]       = {0, 0, 0};
    float    color_distance = 1.f;
};

// A mesh in object space, shared by the instances that place it.
struct Mesh_desc {
    std::vector<float>    positions;  // 3 per vertex
    std::vector<float>    normals;    // 3 per vertex (shading)
    std::vector<float>    uvs;        // 2 per vertex (texture coordinates), or empty
    std::vector<uint32_t> indices;    // 3 per triangle
    std::vector<uint32_t> tri_slot;   // material slot per triangle
};

// A 2-D texture of a material, its texels already decoded for their use (colour: linear
// ACEScg; surface: roughness, metallic), sampled bilinearly or nearest, repeating or clamped,
// at the hit's texture coordinates times scale (texture_sampler.cpp Linear_2D / Nearest_2D).
struct Texture_desc {
    uint32_t           width    = 0;
    uint32_t           height   = 0;
    uint32_t           channels = 0;  // 1 to 3 values per texel in texels
    std::vector<float> texels;
    bool               nearest  = false;
    bool               clamp    = false;
    float              scale[2] = {1.f, 1.f};
};

// A prop: a mesh placed by a row-major object-to-world matrix (translation in the last row, as
// su_entity_set_transformation takes it; points are row vectors times the matrix), the
// rotation its normals turn by, its materials per slot, and whether it is a light.  A light
// prop's emitting medium needs a material of its own (Material::volume_light names one light).
struct Instance_desc {
    uint32_t              mesh      = 0;
    float                 trafo[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    float                 rotation[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // row-major, normals as row vectors
    std::vector<uint32_t> materials;  // slot -> index into Scene_desc::materials
    uint32_t              fallback  = 0;  // material of slots beyond `materials`
    bool                  light     = false;
    // The mesh is the built-in Cube, [-1, 1]^3 in object space: an emitting medium inside it is
    // a light that next-event estimation samples (Cube::sample_volume).
    bool                  cube      = false;
};

// The scene as the host engine collects it (prop_bvh_wrapper.cpp, prop.cpp: props placing
// shapes).  The renderer either flattens every instance into one world-space tree, or -- when
// props share meshes enough for it to pay -- keeps one tree per mesh in object space under a
// top-level tree over the instances (instancing).
struct Scene_desc {
    std::vector<Mesh_desc>          meshes;
    std::vector<Instance_desc>      instances;
    std::vector<shading::Material>  materials;    // Volume materials: medium = 1 + grid medium
    std::vector<Density_grid>       grids;
    std::vector<Grid_medium>        media;
    std::vector<Texture_desc>       textures;     // Material::color_map / surface_map - 1 index this
    float                           environment[3] = {0.f, 0.f, 0.f};  // uniform radiance at infinity
    bool                            environment_light = false;  // also sampled by next-event estimation
    // Two-level trees: -1 when flattening would hold more than four times the triangles of the
    // distinct meshes and over a million triangles; 0 never; 1 always.
    int                             instancing = -1;
};

constexpr uint32_t Max_views = 4096;

struct Camera_desc {
    uint32_t width  = 0;
    uint32_t height = 0;
    float    fov    = 0.f;              // horizontal, radians
    float    rotation[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // rows: camera x, y, z axes in world
    float    position[3] = {0, 0, 0};
};

struct Settings {
    uint32_t min_bounces = 4;   // Russian roulette starts here
    uint32_t max_bounces = 8;
    uint32_t seed        = 0;
    // Light selection (the PTMIS "light_sampling" object): Adaptive splits the selection at the
    // first three vertices (the environment with probability 1, and every light-tree node
    // whose split test passes descended on both sides), Single picks one light everywhere;
    // split_threshold is the reference's splitting_threshold to the fourth power.
    bool     light_split     = true;
    float    split_threshold = 4.096e-5f;
    // Golden ratio sequences for the camera and the first three vertices of a frame rendered in
    // one call (the reference's batch mode); false: independent random samples (progressive).
    bool     golden_ratio = false;
    // Learned path guiding (no counterpart in the reference): at surface vertices the
    // continuation direction comes from the network's vMF mixture with probability
    // guide_fraction, else from the BSDF (one-sample MIS of the two).  The network is trained
    // online: guide_steps Adam steps (learning rate guide_lr) on batches of guide_batch records
    // after each pass of guide_pass_spp samples per pixel, from the first record_depth vertices
    // of every path, until guide_train_spp samples per pixel have been rendered.
    bool     guiding         = false;
    float    guide_fraction  = 0.5f;
    float    metal_fraction  = -1.f;  // at metallic surfaces; negative: guide_fraction
    uint32_t guide_batch     = 1u << 16;
    uint32_t guide_steps     = 16;
    float    guide_lr        = 1e-2f;
    uint32_t record_depth    = 2;
    uint32_t guide_seed      = 7;
    uint32_t guide_pass_spp  = 1;   // samples per pixel between training steps
    uint32_t guide_train_spp = 16;  // samples per pixel after which training stops (0: never)
    uint32_t guide_depth     = 255;  // vertices of depth below this are guided
    // Paths per wave and traversal blocks per SM; 0: chosen by the online autotuner.
    uint32_t wave_paths          = 0;
    uint32_t trace_blocks_per_sm = 0;
    // Waves without media or training are captured once per shape as a CUDA graph and replayed.
    bool cuda_graphs = true;
    // Hero-wavelength spectral transport (no counterpart in the reference, which is RGB): each
    // path carries four wavelengths in [380, 720] nm; one persistent launch renders every view
    // and sample.  For scenes of participating media, emitters and the environment.
    bool spectral = false;
};

struct Stats {
    uint64_t paths          = 0;  // camera samples traced
    uint64_t extension_rays = 0;  // closest-hit rays (camera + continuation)
    uint64_t shadow_rays    = 0;  // any-hit rays
    double   seconds        = 0.0;  // device time of the last render call
    uint32_t overflow       = 0;  // rays dropped by the traversal stack guard (0 expected)
    uint64_t guide_vertices          = 0;    // queue entries the guide network was run for
    double   guide_inference_seconds = 0.0;  // device time of encoding + inference
    uint64_t guide_training_samples  = 0;    // Adam steps x batch
    double   guide_training_seconds  = 0.0;  // device time of training
    uint32_t wave_paths              = 0;    // largest wave of the call (paths)
    uint32_t trace_blocks_per_sm     = 0;    // traversal blocks per SM of its last wave
    uint32_t graph_waves             = 0;    // waves replayed from a captured CUDA graph
    uint32_t instances               = 0;    // instances under a top-level tree (0: flattened)
    uint64_t device_triangles        = 0;    // triangles in the uploaded trees
    uint32_t tracking_capped         = 0;    // medium tracking segments cut at their step cap
};

class Renderer {
  public:
    Renderer();
    ~Renderer();

    int32_t set_scene(Scene_desc const& scene, uint32_t num_threads);
    int32_t set_camera(Camera_desc const& camera);
    // Several views rendered together: a render call traces every view's pixels in the same
    // waves (the same samples per pixel), and resolve() returns their images one after another
    // (view 0's width x height pixels first).  set_camera is the one-view case.
    int32_t set_views(std::vector<Camera_desc> const& views);
    void    set_settings(Settings const& s) { settings_ = s; }

    // Clears the film (start of a frame).
    int32_t start_frame();

    // Traces num_samples samples per pixel, samples first .. first + num_samples - 1 of the
    // frame; sample i of a pixel always uses the same random stream.
    int32_t render(uint32_t first_sample, uint32_t num_samples);

    // Film resolve: rgb / weight per pixel (ACEScg linear), alpha 1, into host rgba floats
    // (the views' images one after another).
    int32_t resolve(float* rgba);

    Stats const& stats() const { return stats_; }

    bool ready() const { return scene_ready_ && camera_ready_; }

    std::string const& error() const { return error_; }

  private:
    struct Device;
    Device*     d_ = nullptr;
    Settings    settings_;
    std::vector<Camera_desc> views_;
    Stats       stats_;
    uint32_t    instances_        = 0;  // of the uploaded scene (Stats::instances)
    uint64_t    device_triangles_ = 0;
    bool        scene_ready_  = false;
    bool        camera_ready_ = false;
    std::string error_;

    int32_t ensure_buffers(uint32_t paths, uint32_t picks_per_path);
    // (scene: the kernels' scene parameters, a type private to render.cu)
    int32_t render_spectral(void const* scene, uint32_t first_sample, uint32_t num_samples);
    int32_t ensure_guide(uint32_t paths);
    int32_t train_guide(uint32_t paths);
    void    clear_graphs();
    void    free_grids();
    int32_t fail_cuda(char const* what, int code);
};

}  // namespace spb::render
