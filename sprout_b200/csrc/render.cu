// Wavefront MIS path tracer (sm_100a): the GPU replacement of the reference's
// rendering::Worker::render + Pathtracer_MIS::integrate loop
// (rendering/rendering_worker.cpp:73-128, rendering/integrator/surface/pathtracer_mis.cpp:95-380).
//
// One "wave" traces k samples for every pixel (k * W * H paths).  Per bounce, three kernels
// run over SoA path state in HBM, joined by queues of path indices:
//   extend  closest hit for the paths in the extension queue (persistent warps, dynamic fetch,
//           the cast traversal of traverse.cuh)
//   shade   per hit: emission reached by the BSDF sample (MIS), bounce limit, Russian
//           roulette, light sample + shadow ray (next-event estimation), BSDF sample; appends
//           surviving paths to the next extension queue and shadow rays to the shadow queue
//           (warp-aggregated atomics)
//   shadow  any hit for the shadow queue; unoccluded light samples add their contribution
// After the last bounce, "gather" splats every sample into the film with the reference's
// Gaussian filter (radius 1, alpha 1.8) as a per-pixel gather over the 3x3 neighbourhood (no
// atomics), adding the wave's sum into a compensated (Kahan) FP32 film; "resolve" divides in
// FP64.
//
// The estimator follows Pathtracer_MIS::integrate: emission seen by the camera at the first
// hit, next-event estimation at every non-emissive vertex weighted by the power heuristic
// (predivided form, integrator_helper.hpp:32-40), the BSDF sample's emitter hit weighted by the
// power heuristic against the light pdf, max_bounces / min_bounces with Russian roulette on
// the largest throughput component (integrator_helper.hpp:42-52).  Light selection and
// sampling are this project's own (power-proportional triangle choice, uniform point), an
// unbiased estimator of the same integral.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

#include "bvh8.hpp"
#include "common.hpp"
#include "ggx_table.hpp"
#include "guide.hpp"
#include "guide_mlp.cuh"
#include "light_tree.hpp"
#include "render.hpp"
#include "spectral.cuh"
#include "tuner.hpp"
#include "traverse.cuh"

namespace spb::render {

namespace {

using shading::V3;
using shading::v3;

__device__ __forceinline__ V3 f3v(float4 a) {
    return v3(a.x, a.y, a.z);
}

constexpr uint32_t Full_mask        = 0xFFFFFFFFu;
constexpr int      Trace_block      = 128;
constexpr int      Shade_block      = 256;
constexpr uint32_t Refill_threshold = 8;
constexpr float    Ray_max_t        = 3.4027715434167032e+38f;
constexpr int      Filter_samples   = 30;
constexpr uint32_t Max_bounce_slots = 64;
constexpr uint32_t Class_surface    = 1;  // Wide_triangle::tri_class of ordinary surfaces
constexpr uint32_t Class_boundary   = 2;  // ... of participating-medium boundaries
constexpr uint32_t Class_instance   = 4;  // ... of top-level leaves (instances)

// Counter block (uint32): per bounce b, at Counter_stride * b + k: k = 0 extension count,
// 1 shadow count, 2 extend fetch, 3 shadow fetch, 4 shadow slots through media (rays to
// emitters), 5 picks of split light selections, 6 split records, 7 picks through media,
// 8 shadow slots through media (rays to the environment); then the overflow counter.
constexpr uint32_t Counter_stride = 16;
constexpr uint32_t Graph_max_paths = 1u << 25;  // largest wave replayed from a CUDA graph
constexpr uint64_t Pick_budget     = 24ull << 30;  // bytes of picks a wave may hold
constexpr uint32_t Counter_words  = Counter_stride * Max_bounce_slots + 4;
constexpr uint32_t Overflow_slot  = Counter_stride * Max_bounce_slots;

// A prop filled with a heterogeneous medium: world -> texture space map, its density grid and
// the grid's majorant cells.
struct Medium_gpu {
    float4        m0, m1, m2;  // rows of the world -> texture-space affine map
    float const*  density;     // nx * ny * nz, x fastest
    float2 const* cells;       // per majorant cell: (min, max) density
    int           nx, ny, nz;
    int           cx, cy, cz;  // majorant cells per axis
    uint32_t      flags;       // bit 0: Nearest filter; bit 1: Repeat address mode
    uint32_t      pad;
    // An emitting grid's temperature (same dimensions as the density) and the emission at 16
    // temperatures (Grid_emission's black-body table); null without a temperature grid.
    float const*  temperature;
    float4 const* blackbody;
    // A two-channel density's second channel, scaling the emission; null for one channel.
    float const*  scale;
    // A colour grid (Grid_color): density is its alpha, rgb its colour; null for a density grid.
    // color_maj: the largest total coefficient any colour gives (-ln 0.01 / distance).
    float const*  rgb[3];
    float         color_distance;
    float         color_maj;
};

// The emission of a temperature grid's material at temperature x: Grid_emission's table of
// 16 samples over [0, 1.2] (volumetric_grid.cpp:140-160), x clamped to the range and
// interpolated linearly (Interpolated_function_1D::operator(), interpolated_function_1d.inl:86-96).
__host__ __device__ inline V3 blackbody_emission(float4 const* table, float x) {
    float const    o = fminf(fmaxf(x, 0.f), 1.2f) * 12.5f;
    uint32_t const i = min(uint32_t(o), 15u);
    float const    t = o - float(i);
    float4 const   a = table[i];
    float4 const   b = table[min(i + 1u, 15u)];
    return v3(a.x + t * (b.x - a.x), a.y + t * (b.y - a.y), a.z + t * (b.z - a.z));
}

// A material texture (Texture_desc): texels as float4 (unused components 0), x fastest.
struct Texture_gpu {
    float4 const* texels;
    int           w, h;
    uint32_t      flags;  // bit 0: nearest filter; bit 1: clamp address mode (else repeat)
    float         su, sv;  // uv scale
    uint32_t      pad[2];
};

// A Cube prop whose emitting medium is a light (Light::Type::Volume and Volume_image,
// light.cpp:101-134; the cube is [-1, 1]^3 in object space, cube.cpp:134-190): its
// object-to-world map, world volume and material, and for a density grid the 3-D distribution
// its points are drawn from with the grid's normalisation (Grid_emission, volumetric_grid.cpp).
struct Volume_light_gpu {
    float4   m0, m1, m2;  // rows: world_k = dot(row_k.xyz, object) + row_k.w
    float    volume;
    uint32_t material;
    uint32_t dist;        // 0: uniform points (homogeneous medium); else 1 + index into emission_dists
    uint32_t medium;      // the density-grid medium (index into media) when dist != 0
    float    pdf_factor;  // voxels / largest absorption coefficient (Grid_emission::pdf_factor_)
    V3       a_norm;      // largest absorption coefficient / absorption coefficient (a_norm_)
    uint32_t color;       // 1: a colour grid (medium), whose absorption at the point sets the radiance
};

// The 3-D distribution of a density grid's emitted luminance (Grid_emission::prepare_sampling
// with Distribution_3D, volumetric_grid.cpp:182-318, distribution_3d.cpp): per voxel its
// probability, and cumulative sums over slices (z), over the rows of each slice and over the
// voxels of each row, each running from 0 to 1.
struct Emission_dist_gpu {
    float const* prob;   // nx * ny * nz, x fastest
    float const* cdf_z;  // nz + 1
    float const* cdf_y;  // nz * (ny + 1)
    float const* cdf_x;  // nz * ny * (nx + 1)
    int          nx, ny, nz;
    uint32_t     repeat;  // the grid's address mode (1: repeat, 0: clamp)
};

struct Scene_gpu {
    uint4 const*              nodes;
    float4 const*             tris;
    float                     hit_margin;
    uint4 const*              tri_info;  // v0, v1, v2, material
    float4 const*             positions;
    float4 const*             normals;
    shading::Material const*  materials;
    float4 const*             light_nodes;  // light tree (light_tree.hpp): 4 per node
    float4 const*             light_cones;  // 3 per light in tree order: bounds for importance
    float4 const*             light_tris;   // 3 per light in tree order: (a, area), e1, (e2, tri)
    uint32_t const*           light_order;  // per triangle: tree order, 0xFFFFFFFF if no light
    uint32_t                  num_lights;
    float4                    env;  // uniform environment radiance; w: its pick probability in NEE
    float const*              e_table;
    Medium_gpu const*         media;  // Material::medium - 1 indexes this
    // Instances: what the traversal reads (two-level trees only) and what shading reads (also
    // the single identity instance of a flattened scene).
    gpu::Instance_trace const* inst_trace;
    struct Instance_shade const* inst_shade;
    uint32_t const*           inst_materials;  // per instance slot: index into materials
    uint32_t                  instanced;       // 1: two-level trees, hit records name instances
    uint32_t*                 tracking_capped;  // counts tracking segments that reached their step cap
    float2 const*             uvs;       // per vertex, parallel to positions
    Texture_gpu const*        textures;  // Material::color_map / surface_map - 1 index this
    // Light selection splits at vertices of depth below split_bounces (0: never, Single light
    // sampling); the split tree walk starts at depth split_depth_bias.
    uint32_t                  split_bounces;
    uint32_t                  split_depth_bias;
    float                     split_scale;  // 3 (1 / t - 1)^2 for the splitting threshold t (split_node)
    // Emitting media that are lights: their light-tree entries (light_tris) hold -1 - index
    // into volume_lights in the first float4's w.
    Volume_light_gpu const*   volume_lights;
    Emission_dist_gpu const*  emission_dists;
};

// What shading reads of an instance: its object-to-world map (rows: world_k =
// dot(row_k.xyz, object) + row_k.w), the rotation of its normals (rows), its mesh's first entry
// in tri_info, its first material slot in inst_materials, and its first entry in light_order
// (0xFFFFFFFF if it is not a light).  A flattened scene has one instance: the identity.
struct Instance_shade {
    float4   o2w[3];
    float4   nrm[3];
    uint32_t tri_base;
    uint32_t mat_base;
    uint32_t light_base;
    uint32_t pad;
};

__device__ __forceinline__ V3 map_point(float4 const* rows, V3 p) {
    return v3(fmaf(rows[0].x, p.x, fmaf(rows[0].y, p.y, fmaf(rows[0].z, p.z, rows[0].w))),
              fmaf(rows[1].x, p.x, fmaf(rows[1].y, p.y, fmaf(rows[1].z, p.z, rows[1].w))),
              fmaf(rows[2].x, p.x, fmaf(rows[2].y, p.y, fmaf(rows[2].z, p.z, rows[2].w))));
}

// A hit triangle in world space: vertices, the shading normals at them (not normalised) and
// its material; tri: its tri_info entry.
struct World_tri {
    V3       a, b, c;
    uint32_t material;
    uint4    tri;
};

// Triangle id of instance inst (a closest-hit record) in world space; with_normals also gives
// the vertex normals.
__device__ __forceinline__ World_tri world_triangle(Scene_gpu const& s, uint32_t inst, uint32_t id,
                                                    V3* normals = nullptr) {
    Instance_shade const& in = s.inst_shade[inst];
    float4 const o2w[3] = {in.o2w[0], in.o2w[1], in.o2w[2]};
    World_tri    w;
    w.tri      = s.tri_info[in.tri_base + id];
    w.a        = map_point(o2w, f3v(s.positions[w.tri.x]));
    w.b        = map_point(o2w, f3v(s.positions[w.tri.y]));
    w.c        = map_point(o2w, f3v(s.positions[w.tri.z]));
    w.material = s.inst_materials[in.mat_base + w.tri.w];
    if (normals) {
        float4 const rows[3] = {in.nrm[0], in.nrm[1], in.nrm[2]};  // w = 0: no translation
        normals[0] = map_point(rows, f3v(s.normals[w.tri.x]));
        normals[1] = map_point(rows, f3v(s.normals[w.tri.y]));
        normals[2] = map_point(rows, f3v(s.normals[w.tri.z]));
    }
    return w;
}


struct Paths {
    float4*   ray_o;  // origin, min_t
    float4*   ray_d;  // direction, max_t
    uint32_t* hit_id;
    uint32_t* hit_inst;  // instance of the hit (two-level trees only)
    float*    hit_t;
    float2*   hit_uv;
    float4*   T;      // throughput, w: pdf of the last BSDF sample
    float4*   L;      // radiance
    float2*   puv;    // position in the pixel
    uint4*    rng;    // PCG32 state (lo, hi), increment (lo, hi)
    uint32_t* info;   // bits 0-7 vertex count, 8-15 bounce depth, 16 treat-as-singular
    float4*   sh_o;
    float4*   sh_d;
    float4*   sh_L;
    float4*   prev_n;  // geometric normal at the last scattering vertex; w 1: medium vertex
    // Second shadow slot: the environment's sample when light selection splits; its
    // contribution accumulates in L2, so that no two kernel threads add to the same radiance.
    float4*   sh2_o;
    float4*   sh2_d;
    float4*   sh2_L;
    // Vertices whose light selection splits into several lights (select_lights): one record per
    // vertex per bounce -- (shadow-ray origin, path) and (first pick, picks, depth, 0) -- and
    // per selected light a pick: (direction, distance) and (contribution, record).  Shadow rays
    // zero the contributions of occluded picks (and scale those through media); k_pick_sum
    // then adds each record's picks in order to L2 (added to L by gather), so that no two
    // kernel threads ever add to the same radiance and the sum does not depend on scheduling.
    float4*   split_o;
    uint4*    split_m;
    float4*   pick_d;
    float4*   pick_c;
    float4*   L2;
    // Path guiding, indexed by position in the current extension queue: the network inputs as
    // BF16 tiles of 128 entries in the tensor cores' operand order (guide_in), the predicted
    // mixture (guide_out, Mixture_floats per entry) and whether the entry is guided (guide_ok).
    // Indexed by path: the training records of its first record_depth vertices (5 float4 each:
    // position and normal x | normal yz, wo xy | wo z, wi | throughput | radiance mark, w = 1
    // once marked) and the record awaiting its radiance mark.
    __nv_bfloat16* guide_in;
    float*    guide_out;
    uint8_t*  guide_ok;
    float4*   rec;
    uint32_t* open_record;
};

// The instance of a path's closest hit (the only instance of a flattened scene).
__device__ __forceinline__ uint32_t hit_instance(Scene_gpu const& s, Paths const& p, uint32_t path) {
    return s.instanced ? p.hit_inst[path] : 0u;
}

constexpr int Record_float4 = 5;

// The guide's mixture per queue entry: 8 float4 of unit mean and concentration, the 8 lobe
// weights, then the 8 weights times their lobes' vMF normalisation
// kappa / (2 pi (1 - e^{-2 kappa})), so that a density evaluation takes one exponential per lobe.
constexpr int Mixture_floats = 48;

// Shadow-queue entries are path indices (the path's first shadow slot), path indices with
// Second_shadow (its second slot: the environment's sample of a split selection), or pick
// indices with Pick_shadow (an emitter of a split selection that chose several).
constexpr uint32_t Pick_shadow   = 0x80000000u;
constexpr uint32_t Second_shadow = 0x40000000u;
constexpr uint32_t Entry_index   = 0x3FFFFFFFu;

struct Cam {
    float3   left_top;
    float3   d_x;
    float3   d_y;
    float3   r0, r1, r2;
    float3   pos;
    uint32_t w, h;
};

struct Wave {
    uint32_t first_sample;  // frame sample index of slot 0
    uint32_t samples;       // k samples per pixel in this wave
    uint32_t seed;
    uint32_t min_bounces;
    uint32_t max_bounces;
    // Golden ratio sampling of the camera and the first Golden_bounces vertices (see
    // golden_1d): the frame's samples per pixel (0: independent random samples) and the sorted
    // table of frac(j / phi) * 2^32, j < golden_n.
    uint32_t        golden_n;
    uint32_t const* golden_sorted;
    uint32_t guiding;         // 1: sample the guide's mixture at surface vertices
    float    guide_fraction;  // its share of continuation directions
    float    metal_fraction;  // the same at metallic (pure GGX) surfaces
    uint32_t record_depth;    // vertices per path recorded for training (0: none)
    uint32_t guide_depth;     // vertices of depth below this are guided
    float4   bounds_lo;       // scene box, for the guide's position encoding
    float4   bounds_inv;      // 1 / its extent
};

// A wave's launch parameters, which the kernels read from device memory: the host writes them
// (pinned) and copies them before each wave, so that one captured CUDA graph replays every wave
// of the same shape.
//
// A render covers one or more views (cameras with their own resolution), their bordered pixel
// ranges concatenated into one sample space of `pixels` entries: view v owns [view_offsets[v],
// view_offsets[v + 1]) and its film pixels [film_offsets[v], film_offsets[v + 1]).
struct Launch {
    Cam const*      cams;
    uint32_t const* view_offsets;
    uint32_t const* film_offsets;
    uint32_t        num_views;
    uint32_t        pixels;  // bordered pixels of all views
    Wave            wave;
};

// The view owning entry x of a prefix table offsets[0 .. n] (offsets[0] = 0).
__device__ __forceinline__ uint32_t view_of(uint32_t const* offsets, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;  // offsets[lo] <= x < offsets[hi]
    while (hi - lo > 1) {
        uint32_t const mid = (lo + hi) >> 1;
        if (__ldg(offsets + mid) <= x) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// ---- PCG32 (O'Neill 2014), seeded as rnd::Generator::start (base/random/generator.inl) ----
__device__ __forceinline__ uint32_t pcg_next(uint64_t& state, uint64_t inc) {
    uint64_t const old = state;
    state              = old * 6364136223846793005ull + (inc | 1ull);
    uint32_t const xrs = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t const rot = uint32_t(old >> 59u);
    return (xrs >> rot) | (xrs << ((0u - rot) & 31u));
}

struct Rng {
    uint64_t state;
    uint64_t inc;

    __device__ void start(uint64_t seed, uint64_t sequence) {
        state = 0;
        inc   = (sequence << 1u) | 1u;
        pcg_next(state, inc);
        state += seed;
        pcg_next(state, inc);
    }

    __device__ float uniform() {
        uint32_t const bits = (pcg_next(state, inc) & 0x007FFFFFu) | 0x3F800000u;
        return __uint_as_float(bits) - 1.f;
    }

    __device__ void load(uint4 s) {
        state = (uint64_t(s.y) << 32) | s.x;
        inc   = (uint64_t(s.w) << 32) | s.z;
    }

    __device__ uint4 save() const {
        return make_uint4(uint32_t(state), uint32_t(state >> 32), uint32_t(inc), uint32_t(inc >> 32));
    }
};


// ---- golden ratio sampling (sampler::Golden_ratio, sampler_golden_ratio.cpp:21-73) ----
// In batch rendering the reference samples the camera and, at the first three vertices of a
// path, light selection, light points and BSDF directions from golden ratio sequences
// (Pathtracer_MIS::material_sampler / light_sampler, pathtracer_mis.cpp:403-417): per pixel and
// dimension the frame's n samples are frac(r + j / phi), j < n, with a random offset r, put in
// a random order; 2-D dimensions pair the same sequence, sorted, with a second one
// (golden_ratio in sample_distribution.inl, after Schretter, Kobbelt and Dehaye 2012).  Every
// sample of a pixel thus lands in its own stratum of each dimension.  Here any sample is
// computed directly from its index: in 32-bit fixed point (2^32 / phi rounds to 2654435769),
// with a keyed bijection of [0, n) as the per-pixel shuffle (the reference shuffles with its
// pixel's random stream) and, for the sorted first coordinates, a table of the sequence
// without offset in ascending order, which the offset rotates.
constexpr uint32_t Golden_step    = 2654435769u;
constexpr uint32_t Golden_bounces = 3;  // Pathtracer_MIS::Num_dedicated_samplers

// A bijection of [0, n) chosen by key: an invertible mix of the bits below n's next power of
// two (odd multiplications, xor-shifts and additions, each a bijection of that range),
// repeated until the value falls below n (cycle walking).
__device__ __forceinline__ uint32_t permute(uint32_t i, uint32_t n, uint32_t key) {
    uint32_t mask = n - 1u;
    mask |= mask >> 1;
    mask |= mask >> 2;
    mask |= mask >> 4;
    mask |= mask >> 8;
    mask |= mask >> 16;
    uint32_t const m1 = (key * 2u + 1u) | 1u;
    uint32_t const a1 = key >> 11;
    do {
        i = ((i ^ (key >> 5)) * m1) & mask;
        i ^= i >> 3;
        i = (i + a1) & mask;
        i = (i * 0x2C9277B5u) & mask;
        i ^= (i & mask) >> 5;
        i = ((i ^ (key >> 19)) * 0x85EBCA77u) & mask;
        i ^= i >> 2;
    } while (i >= n);
    return i;
}

// Offset and shuffle key of a pixel's golden ratio dimension (its own PCG32 stream).
__device__ __forceinline__ void golden_stream(uint32_t seed, uint32_t pixel, uint32_t dim, uint32_t& off0,
                                              uint32_t& off1, uint32_t& key) {
    uint64_t       state = 0;
    uint64_t const inc   = ((uint64_t(pixel) << 6 | dim) << 1) | 1u;
    pcg_next(state, inc);
    state += uint64_t(seed) ^ 0x9E3779B97F4A7C15ull;
    pcg_next(state, inc);
    off0 = pcg_next(state, inc);
    off1 = pcg_next(state, inc);
    key  = pcg_next(state, inc);
}

__device__ __forceinline__ float fixed_to_unit(uint32_t x) {
    return float(x >> 8) * (1.f / 16777216.f);
}

// Sample s of 1-D dimension dim of a pixel.
__device__ __forceinline__ float golden_1d(Wave const& w, uint32_t pixel, uint32_t s, uint32_t dim) {
    uint32_t off0, off1, key;
    golden_stream(w.seed, pixel, dim, off0, off1, key);
    uint32_t const j = permute(s, w.golden_n, key);
    return fixed_to_unit(off0 + j * Golden_step);
}

// Sample s of 2-D dimension dim of a pixel.
__device__ __forceinline__ float2 golden_2d(Wave const& w, uint32_t pixel, uint32_t s, uint32_t dim) {
    uint32_t off0, off1, key;
    golden_stream(w.seed, pixel, dim, off0, off1, key);
    uint32_t const n = w.golden_n;
    uint32_t const i = permute(s, n, key);
    // First coordinate: the i-th smallest of frac(off0 + j / phi), j < n -- the sorted table
    // rotated to start at c, the first entry that wraps past 1 when off0 is added.
    uint64_t const wrap = (1ull << 32) - off0;
    uint32_t       lo = 0, hi = n;
    while (lo < hi) {
        uint32_t const mid = (lo + hi) >> 1;
        if (uint64_t(__ldg(w.golden_sorted + mid)) < wrap) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    uint32_t k = lo + i;
    k      = k >= n ? k - n : k;
    return make_float2(fixed_to_unit(__ldg(w.golden_sorted + k) + off0), fixed_to_unit(off1 + i * Golden_step));
}

// Golden ratio dimensions: 2-D 0 the pixel position, the light point of the l-th selected light
// at vertex depth d 1 + 4 d + l for l < 3 and 64 + 64 d + l beyond (the reference gives each
// light of a split selection its own dimension, pathtracer_mis.cpp:298-318), 1 + 4 d + 3 the
// BSDF (or guide) direction; 1-D 16 + 4 d the light selection, 16 + 4 d + 3 the BSDF lobe (or
// guide lobe), 32 + d the choice between guide and BSDF.
__device__ __forceinline__ uint32_t golden_light_2d(uint32_t depth, uint32_t l) {
    return l < 3u ? 1u + 4u * depth + l : 64u + 64u * depth + l;
}
__device__ __forceinline__ uint32_t golden_bsdf_2d(uint32_t depth) { return 1u + 4u * depth + 3u; }
__device__ __forceinline__ uint32_t golden_light_1d(uint32_t depth, int k) { return 16u + 4u * depth + uint32_t(k); }
__device__ __forceinline__ uint32_t golden_bsdf_1d(uint32_t depth) { return 16u + 4u * depth + 3u; }
__device__ __forceinline__ uint32_t golden_choice_1d(uint32_t depth) { return 32u + depth; }

// Ray origin offset off a surface (Waechter and Binder, "A Fast and Robust Method for
// Avoiding Self-Intersection", Ray Tracing Gems 2019, ch. 6), n pointing to the side the ray
// leaves on.
__device__ __forceinline__ V3 offset_ray(V3 p, V3 n) {
    float const origin      = 1.f / 32.f;
    float const float_scale = 1.f / 65536.f;
    float const int_scale   = 256.f;
    int const   ox          = int(int_scale * n.x);
    int const   oy          = int(int_scale * n.y);
    int const   oz          = int(int_scale * n.z);
    float const px = __int_as_float(__float_as_int(p.x) + (p.x < 0.f ? -ox : ox));
    float const py = __int_as_float(__float_as_int(p.y) + (p.y < 0.f ? -oy : oy));
    float const pz = __int_as_float(__float_as_int(p.z) + (p.z < 0.f ? -oz : oz));
    return v3(fabsf(p.x) < origin ? p.x + float_scale * n.x : px,
              fabsf(p.y) < origin ? p.y + float_scale * n.y : py,
              fabsf(p.z) < origin ? p.z + float_scale * n.z : pz);
}

__device__ __forceinline__ float power_heuristic(float f, float g) {
    float const f2 = f * f;
    return f2 / (f2 + g * g);
}

// Warp-aggregated append: returns this lane's slot in the queue.
__device__ __forceinline__ uint32_t append(uint32_t* counter, bool want) {
    uint32_t const mask = __ballot_sync(__activemask(), want);
    if (!want) {
        return 0;
    }
    uint32_t const lane   = threadIdx.x & 31u;
    uint32_t const leader = __ffs(mask) - 1;
    uint32_t       base   = 0;
    if (lane == leader) {
        base = atomicAdd(counter, __popc(mask));
    }
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// Samples are taken over the image plus a border of the filter's integer radius, whose
// filtered contributions reach the edge pixels (the reference's tile queue extends the edge
// tiles by filter_radius_int, tile_queue.cpp:54-68; sample streams per bordered pixel as in
// rendering_worker.cpp:93-104).
constexpr int Film_border = 1;

// ---- generate: camera rays (Perspective::generate_ray, camera_perspective.cpp:47-80) ----
__global__ void k_generate(Launch const* __restrict__ launch, Paths p, uint32_t* queue, uint32_t* counters,
                           uint32_t num_paths) {
    Wave const     wave = launch->wave;
    uint32_t const i    = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        counters[0] = num_paths;
    }
    if (i >= num_paths) {
        return;
    }
    uint32_t const pixels = launch->pixels;
    uint32_t const pixel  = i % pixels;
    uint32_t const slot   = i / pixels;
    uint32_t const view   = view_of(launch->view_offsets, launch->num_views, pixel);
    Cam const      cam    = launch->cams[view];
    uint32_t const local  = pixel - launch->view_offsets[view];
    uint32_t const bw     = cam.w + 2 * Film_border;
    int const      x      = int(local % bw) - Film_border;
    int const      y      = int(local / bw) - Film_border;

    // A view's sample streams depend on its own pixel index and size only, so that a view
    // rendered with others traces the paths it would trace alone.
    uint32_t const view_pixels = launch->view_offsets[view + 1] - launch->view_offsets[view];
    Rng            rng;
    rng.start(wave.seed, uint64_t(local) + uint64_t(wave.first_sample + slot) * view_pixels);
    float u = rng.uniform();
    float v = rng.uniform();
    if (wave.golden_n) {
        float2 const g = golden_2d(wave, local, wave.first_sample + slot, 0);
        u              = g.x;
        v              = g.y;
    }

    float const cx = float(x) + u;
    float const cy = float(y) + v;
    float3 d = make_float3(cam.left_top.x + cx * cam.d_x.x + cy * cam.d_y.x,
                           cam.left_top.y + cx * cam.d_x.y + cy * cam.d_y.y,
                           cam.left_top.z + cx * cam.d_x.z + cy * cam.d_y.z);
    float const inv = rsqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
    d.x *= inv;
    d.y *= inv;
    d.z *= inv;
    float3 const w = make_float3(d.x * cam.r0.x + d.y * cam.r1.x + d.z * cam.r2.x,
                                 d.x * cam.r0.y + d.y * cam.r1.y + d.z * cam.r2.y,
                                 d.x * cam.r0.z + d.y * cam.r1.z + d.z * cam.r2.z);

    p.ray_o[i] = make_float4(cam.pos.x, cam.pos.y, cam.pos.z, 0.f);
    p.ray_d[i] = make_float4(w.x, w.y, w.z, Ray_max_t);
    p.T[i]     = make_float4(1.f, 1.f, 1.f, 0.f);
    p.L[i]     = make_float4(0.f, 0.f, 0.f, 0.f);
    p.L2[i]    = make_float4(0.f, 0.f, 0.f, 0.f);
    p.puv[i]   = make_float2(u, v);
    p.rng[i]   = rng.save();
    p.info[i]  = 1u << 16;  // vertex 0, depth 0, treat as singular
    queue[i]   = i;
    if (wave.record_depth) {
        p.open_record[i] = 0xFFFFFFFFu;
        for (uint32_t j = 0; j < wave.record_depth; ++j) {
            p.rec[(size_t(i) * wave.record_depth + j) * Record_float4 + 4] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

// Where k_trace puts unoccluded shadow rays of a scene with media (for k_transmit): slot
// entries into queue (rays to emitters from the front, counted by count; rays to the
// environment from the back, entry capacity - 1 downwards, counted by env_count), picks into
// pick_queue.
struct Transmit_out {
    uint32_t* queue;
    uint32_t* count;
    uint32_t* env_count;
    uint32_t  capacity;
    uint32_t* pick_queue;
    uint32_t* pick_count;
};

// ---- extend / shadow: persistent traversal over a queue of path indices ----
// Any_hit: shadow rays.  Media: the scene has participating media -- shadow rays ignore
// medium boundaries and unoccluded ones go to the transmittance queue instead of adding
// their contribution directly.
// Instances: the scene is a top-level tree over instances of per-mesh trees.
template <bool Any_hit, bool Media = false, bool Instances = false>
__global__ void __launch_bounds__(Trace_block)
    k_trace(Scene_gpu s, Paths p, uint32_t const* __restrict__ queue,
            uint32_t const* __restrict__ count, uint32_t* fetch, uint32_t* overflow,
            Transmit_out tq = Transmit_out{}) {
    uint32_t const num  = *count;
    uint32_t const lane = threadIdx.x & 31u;
    uint32_t const lt   = (1u << lane) - 1u;

    gpu::Ray_state      r;
    gpu::Traversal      tv;
    gpu::Instance_state is;
    uint2               stack[gpu::Stack_size];
    uint32_t       path      = 0;
    bool           active    = false;
    bool           exhausted = false;

    while (true) {
        uint32_t const idle = __ballot_sync(Full_mask, !active);
        if (exhausted && idle == Full_mask) {
            break;
        }
        if (!exhausted && __popc(idle) >= int(Refill_threshold)) {
            uint32_t const n      = __popc(idle);
            uint32_t const leader = __ffs(idle) - 1;
            uint32_t       base   = 0;
            if (lane == leader) {
                base = atomicAdd(fetch, n);
            }
            base = __shfl_sync(Full_mask, base, leader);
            if (uint64_t(base) + n >= num) {
                exhausted = true;
            }
            if (!active) {
                uint32_t const mine = base + __popc(idle & lt);
                if (mine < num) {
                    path = queue[mine];
                    if (Any_hit) {
                        uint32_t const e = path & Entry_index;
                        if (path & Pick_shadow) {
                            uint32_t const rec = __float_as_uint(p.pick_c[e].w);
                            float4 const   o   = p.split_o[rec];
                            gpu::start_ray(r, tv, make_float4(o.x, o.y, o.z, 0.f), p.pick_d[e]);
                        } else if (path & Second_shadow) {
                            gpu::start_ray(r, tv, p.sh2_o[e], p.sh2_d[e]);
                        } else {
                            gpu::start_ray(r, tv, p.sh_o[e], p.sh_d[e]);
                        }
                    } else {
                        gpu::start_ray(r, tv, p.ray_o[path], p.ray_d[path]);
                    }
                    if constexpr (Instances) {
                        gpu::start_instances(r, is);
                    }
                    active = true;
                }
            }
        }
        if (!active) {
            continue;
        }
        if (gpu::traversal_step<Any_hit, Media, Instances>(r, tv, stack, s.nodes, s.tris, s.hit_margin,
                                                            overflow, Class_boundary, &is,
                                                            s.inst_trace)) {
            if (Any_hit) {
                uint32_t const e = path & Entry_index;
                if (r.best_id == gpu::Miss) {
                    if (Media) {
                        // Through media: picks to their own queue; slot rays to the environment
                        // fill the slot queue from its back, the others from its front, so that
                        // k_transmit's warps walk rays of one kind (their lengths through a
                        // medium differ widely).
                        if (path & Pick_shadow) {
                            tq.pick_queue[atomicAdd(tq.pick_count, 1u)] = path;
                        } else if (((path & Second_shadow) ? p.sh2_d[e].w : p.sh_d[e].w) >= Ray_max_t) {
                            tq.queue[tq.capacity - 1u - atomicAdd(tq.env_count, 1u)] = path;
                        } else {
                            tq.queue[atomicAdd(tq.count, 1u)] = path;
                        }
                    } else if (!(path & Pick_shadow)) {
                        bool const   second = path & Second_shadow;
                        float4 const c      = second ? p.sh2_L[e] : p.sh_L[e];
                        float4* const Lp    = second ? p.L2 : p.L;
                        float4       l      = Lp[e];
                        l.x += c.x;
                        l.y += c.y;
                        l.z += c.z;
                        Lp[e] = l;
                    }
                } else if (path & Pick_shadow) {
                    // occluded: the pick adds nothing
                    float* const c = reinterpret_cast<float*>(p.pick_c + e);
                    c[0] = 0.f;
                    c[1] = 0.f;
                    c[2] = 0.f;
                }
            } else {
                p.hit_id[path] = r.best_id;
                p.hit_t[path]  = r.tbest;
                p.hit_uv[path] = make_float2(r.u, r.v);
                if constexpr (Instances) {
                    p.hit_inst[path] = is.best_inst;
                }
            }
            active = false;
        }
    }
}

// Small step past a hit distance for a ray that continues through a null boundary
// (scene::offset_f): 256 ulps, or 2^-16 near zero.
__device__ __forceinline__ float offset_f(float t) {
    return t < (1.f / 32.f) ? t + (1.f / 65536.f) : __int_as_float(__float_as_int(t) + 256);
}

constexpr float    Abort_epsilon  = 7.5e-4f;  // Tracking::Abort_epsilon, tracking.hpp:71

__device__ __forceinline__ uint32_t pack_info(uint32_t vtx, uint32_t depth, bool singular,
                                              uint32_t medium) {
    return (vtx & 0xFFu) | ((depth & 0xFFu) << 8) | (singular ? (1u << 16) : 0u) | (medium << 17);
}

// ---- light tree (light_tree.hpp): importance, sampling and pdf ----
// cos(max(a - b, 0)) and sin(max(a - b, 0)) from the cosines and sines of a and b.
__device__ __forceinline__ float cos_sub_clamped(float ca, float cb, float sa, float sb) {
    return ca > cb ? 1.f : ca * cb + sa * sb;
}
__device__ __forceinline__ float sin_sub_clamped(float ca, float cb, float sa, float sb) {
    return ca > cb ? 0.f : sa * cb - ca * sb;
}

// Importance of a light cluster seen from p (normal n, or the whole sphere of directions for a
// medium vertex): power / squared distance (not closer than half the bounding radius) times
// the best cosines the bounding sphere and normal cone allow at the emitter and the receiver
// (Estevez and Kulla 2018, eq. 3; the reference's importance(), light_tree.cpp:27-62).
// Never 0, so that every light keeps a positive probability.
__device__ float light_importance(float4 sphere, float4 cone, float power, V3 p, V3 n,
                                  bool total_sphere) {
    V3 const    v  = v3(sphere.x - p.x, sphere.y - p.y, sphere.z - p.z);
    float const d2 = fmaxf(shading::dot(v, v), 1e-30f);
    float const il = rsqrtf(d2);
    V3 const    w  = il * v;  // towards the cluster
    float const su = fminf(sphere.w * il, 1.f);
    float const cu = sqrtf(fmaxf(1.f - su * su, 0.f));
    // emitter side: angle between the cone axis and the direction from the cluster to p
    float       ce = 1.f;
    if (cone.w > -1.f) {
        float const ca = -(cone.x * w.x + cone.y * w.y + cone.z * w.z);
        float const sa = sqrtf(fmaxf(1.f - ca * ca, 0.f));
        float const so = sqrtf(fmaxf(1.f - cone.w * cone.w, 0.f));
        float const c1 = cos_sub_clamped(ca, cone.w, sa, so);
        float const s1 = sin_sub_clamped(ca, cone.w, sa, so);
        ce             = fmaxf(cos_sub_clamped(c1, cu, s1, su), 0.f);
    }
    // receiver side
    float cr = 1.f;
    if (!total_sphere) {
        float const ci = shading::dot(n, w);
        float const si = sqrtf(fmaxf(1.f - ci * ci, 0.f));
        cr             = fmaxf(cos_sub_clamped(ci, cu, si, su), 0.f);
    }
    float const dist = fmaxf(d2, 0.25f * sphere.w * sphere.w);
    return fmaxf(power * ce * cr / dist, 1e-30f);
}

// Light-tree nodes: 4 float4 each (light_tree.hpp): (centre, radius), (axis, cos spread),
// (power, first, count, middle), (variance, lights, 0, 0).
constexpr uint32_t Light_node_stride = 4;
constexpr uint32_t Env_pick          = 0xFFFFFFFFu;  // a pick of the environment

__device__ __forceinline__ float node_importance(Scene_gpu const& s, uint32_t node, V3 p, V3 n,
                                                 bool total_sphere) {
    float4 const* nd = s.light_nodes + Light_node_stride * node;
    return light_importance(nd[0], nd[1], nd[2].x, p, n, total_sphere);
}

__device__ __forceinline__ float emitter_importance(Scene_gpu const& s, uint32_t l, V3 p, V3 n,
                                                    bool total_sphere) {
    return light_importance(s.light_cones[3 * l], s.light_cones[3 * l + 1], s.light_cones[3 * l + 2].x,
                            p, n, total_sphere);
}

// Whether light selection at p descends into both children of a node (Node::split,
// light_tree.cpp:197-224; Estevez and Kulla 2018, sec. 5).  With g = 1 / x^2 for x uniform
// between the near and far side of the node's bounding sphere, a = max(d - r, 0.001) and
// b = d + r: E[g] = 1 / (a b), E[g^2] = (b^3 - a^3) / (3 (b - a) a^3 b^3), V[g] = E[g^2] - E[g]^2;
// with the variance ve and mean ee of the node's light powers, the estimate's variance is
// s2 = ve V[g] + ve E[g]^2 + ee^2 V[g], and the node splits when 1 / (1 + sqrt(s2)) falls to
// the threshold t, i.e. s2 >= S = (1 / t - 1)^2.  Multiplied by 3 (b - a) a^3 b^3 > 0 (under
// which V[g] becomes (b - a)^3 and E[g]^2 becomes 3 (b - a) a b) and divided by b - a, the
// test needs no division: (ve + ee^2) (b - a)^2 + 3 ve a b >= 3 S a^3 b^3.  b = a (a point
// light at a distance) does not split, as the reference's undefined V[g] does not.
// The host stores with each node the squared distance from its centre beyond which the test
// cannot pass (0: nowhere; split_radius2), which most shading points are beyond.
__device__ __forceinline__ bool split_node(Scene_gpu const& s, uint32_t node, V3 p) {
    float4 const* nd  = s.light_nodes + Light_node_stride * node;
    float4 const  var = nd[3];  // (ve, lights, ve + ee^2, split radius^2)
    if (!(var.w > 0.f)) {
        return false;
    }
    float4 const sph = nd[0];
    V3 const     v   = v3(p.x - sph.x, p.y - sph.y, p.z - sph.z);
    float const  d2  = shading::dot(v, v);
    if (d2 >= var.w) {
        return false;
    }
    float const   d   = fminf(sqrtf(d2), 1e6f);
    float const   a   = fmaxf(d - sph.w, 0.001f);
    float const   b   = d + sph.w;
    float const   ab  = a * b;
    float const   bma = b - a;
    return bma > 0.f && var.z * bma * bma + 3.f * var.x * ab >= s.split_scale * (ab * ab * ab);
}

// One light of a selection: its tree-order index (or Env_pick) and the probability with which
// the selection contains it.
struct Light_pick {
    uint32_t light;
    float    pdf;
};

// Chooses a leaf light in proportion to the importances of the leaf's lights.
__device__ __forceinline__ Light_pick pick_in_leaf(Scene_gpu const& s, uint32_t first, uint32_t count,
                                                   V3 p, V3 n, bool total_sphere, float r) {
    float w[Light_leaf_size];
    float sum = 0.f;
    for (uint32_t k = 0; k < Light_leaf_size; ++k) {
        w[k] = k < count ? emitter_importance(s, first + k, p, n, total_sphere) : 0.f;
        sum += w[k];
    }
    float    acc    = 0.f;
    uint32_t chosen = count - 1;
    for (uint32_t k = 0; k + 1 < count; ++k) {
        acc += w[k];
        if (r * sum < acc) {
            chosen = k;
            break;
        }
    }
    return {first + chosen, w[chosen] / sum};
}

// Light selection at p (normal n; total_sphere for medium vertices) with the random number r:
// Tree::random_light (light_tree.cpp:363-461).  Without splitting one light: the environment
// with probability env.w, else an emitter found by walking the tree, each step choosing a child
// in proportion to its importance.  With splitting (the first vertices of Adaptive light
// sampling): the environment with probability 1, and the tree walked from depth
// split_depth_bias, descending into both children of every node that split_node passes while
// above Max_split_depth (a leaf so reached gives all its lights); below the first node that does
// not split, the walk chooses as before, with the random number it carried.  Hands each light to
// emit(index, pick) (at most Max_light_picks, the host having bounded the tree's picks so),
// stopping early when emit returns false, and returns the number emitted.
template <class Emit>
__device__ uint32_t walk_lights(Scene_gpu const& s, V3 p, V3 n, bool total_sphere, float r, bool split, Emit&& emit) {
    uint32_t m     = 0;
    float    ip    = 0.f;
    uint32_t depth = Max_split_depth;
    if (split) {
        depth = s.split_depth_bias;
        if (s.env.w > 0.f && !emit(m++, Light_pick{Env_pick, 1.f})) {
            return m;
        }
    } else {
        ip = s.env.w;
        if (r < ip) {
            emit(m++, Light_pick{Env_pick, ip});
            return m;
        }
    }
    if (s.num_lights == 0) {
        return m;
    }
    struct Walk {
        uint32_t node;
        uint32_t depth;
        float    pdf;
        float    r;
    };
    Walk     stack[Max_split_depth + 1];
    uint32_t top = 0;
    Walk     t{0u, depth, 1.f - ip, fminf((r - ip) / (1.f - ip), 0x1.fffffep-1f)};
    for (int step = 0; step < 4096; ++step) {
        float4 const   meta     = s.light_nodes[Light_node_stride * t.node + 2];
        uint32_t const first    = __float_as_uint(meta.y);
        uint32_t const count    = __float_as_uint(meta.z);
        bool const     do_split = t.depth < Max_split_depth && split_node(s, t.node, p);
        if (count == 0) {
            if (do_split) {
                if (top < Max_split_depth + 1) {
                    stack[top++] = {first + 1, t.depth + 1, t.pdf, t.r};
                }
                t.node = first;
                ++t.depth;
            } else {
                float const w0 = node_importance(s, first, p, n, total_sphere);
                float const w1 = node_importance(s, first + 1, p, n, total_sphere);
                float const p0 = w0 / (w0 + w1);
                if (t.r < p0) {
                    t.node = first;
                    t.pdf *= p0;
                    t.r = fminf(t.r / p0, 0x1.fffffep-1f);
                } else {
                    t.node = first + 1;
                    t.pdf *= 1.f - p0;
                    t.r = fminf((t.r - p0) / (1.f - p0), 0x1.fffffep-1f);
                }
                t.depth = Max_split_depth;
            }
            continue;
        }
        if (do_split) {
            for (uint32_t k = 0; k < count && m < Max_light_picks; ++k) {
                if (!emit(m++, Light_pick{first + k, t.pdf})) {
                    return m;
                }
            }
        } else if (m < Max_light_picks) {
            Light_pick const pk = pick_in_leaf(s, first, count, p, n, total_sphere, t.r);
            if (!emit(m++, Light_pick{pk.light, pk.pdf * t.pdf})) {
                return m;
            }
        }
        if (top == 0) {
            break;
        }
        t = stack[--top];
    }
    return m;
}

// select_lights into an array (at most Max_light_picks entries; one without splitting).
__device__ __forceinline__ uint32_t select_lights(Scene_gpu const& s, V3 p, V3 n, bool total_sphere, float r,
                                                  bool split, Light_pick* out) {
    return walk_lights(s, p, n, total_sphere, r, split, [&](uint32_t k, Light_pick pk) {
        out[k] = pk;
        return true;
    });
}

// Probability that select_lights from (p, n) includes the light at tree position order
// (Tree::pdf, light_tree.cpp:564-640): 1 through every split, the children's importances
// below.
__device__ float light_pick_pdf(Scene_gpu const& s, V3 p, V3 n, bool total_sphere, uint32_t order,
                                bool split) {
    float    pdf   = split ? 1.f : 1.f - s.env.w;
    uint32_t node  = 0;
    uint32_t depth = split ? s.split_depth_bias : Max_split_depth;
    for (int level = 0; level < 64; ++level, ++depth) {
        float4 const   meta     = s.light_nodes[Light_node_stride * node + 2];
        uint32_t const first    = __float_as_uint(meta.y);
        uint32_t const count    = __float_as_uint(meta.z);
        bool const     do_split = depth < Max_split_depth && split_node(s, node, p);
        if (count != 0) {
            if (do_split) {
                return pdf;
            }
            float sum  = 0.f;
            float mine = 0.f;
            for (uint32_t k = 0; k < count && k < Light_leaf_size; ++k) {
                uint32_t const l = first + k;
                float const    w = emitter_importance(s, l, p, n, total_sphere);
                sum += w;
                mine = l == order ? w : mine;
            }
            return pdf * (mine / sum);
        }
        bool const left = order < __float_as_uint(meta.w);
        if (!do_split) {
            float const w0 = node_importance(s, first, p, n, total_sphere);
            float const w1 = node_importance(s, first + 1, p, n, total_sphere);
            float const p0 = w0 / (w0 + w1);
            pdf *= left ? p0 : 1.f - p0;
            depth = Max_split_depth;
        }
        node = left ? first : first + 1;
    }
    return 0.f;
}

// Light sample for next-event estimation seen from ps (normal n; total_sphere for medium
// vertices) from a selected light: a uniform point on it (or a uniform direction for the
// environment), the solid-angle pdf times the selection probability.  False if the sample is
// unusable (grazing or behind a one-sided emitter, Mesh::sample in triangle_mesh.cpp:462-516).
struct Light_sample {
    V3    dir;
    float dist;
    float pdf;
    V3    radiance;
};

// Light selection splits at the first Split_bounces vertices with the reference's Adaptive
// light sampling (Pathtracer_MIS::splitting, pathtracer_mis.cpp:419-422): the environment is
// sampled with probability 1 there, beside the emitters the split tree walk selects, each with
// a shadow ray.  The reference decides this from the depth at the vertex for next-event
// estimation but from the depth after the bounce when it weighs the light hit (connect_light
// runs after ++ray.depth), and this renderer does the same so that images agree.
constexpr uint32_t Split_bounces = 3;  // Pathtracer_MIS::Num_dedicated_samplers

// Index i in [0, n) with cdf[i] <= r < cdf[i + 1] for r in [0, 1) (cdf[0] = 0, cdf[n] = 1),
// and where r falls inside that bucket.
__device__ __forceinline__ int cdf_bucket(float const* cdf, int n, float r, float& frac) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        int const mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) <= r) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    float const c0 = __ldg(cdf + lo);
    float const c1 = __ldg(cdf + lo + 1);
    frac           = c1 > c0 ? fminf((r - c0) / (c1 - c0), 0.99999994f) : 0.5f;
    return lo;
}

// A voxel drawn in proportion to its probability and a uniform point in it (slice, then row,
// then voxel, as Distribution_3D::sample_continuous, distribution_3d.cpp:46-55); returns the
// voxel's probability (0 if none can be drawn), its index and the point in texture space.
__device__ float sample_emission(Emission_dist_gpu const& e, float r1, float r2, float r3, uint32_t& voxel,
                                 V3& uvw) {
    float      fz, fy, fx;
    int const  z = cdf_bucket(e.cdf_z, e.nz, r3, fz);
    int const  y = cdf_bucket(e.cdf_y + size_t(z) * (e.ny + 1), e.ny, r2, fy);
    int const  x = cdf_bucket(e.cdf_x + (size_t(z) * e.ny + y) * (e.nx + 1), e.nx, r1, fx);
    voxel        = uint32_t((size_t(z) * e.ny + y) * e.nx + x);
    uvw          = v3((float(x) + fx) / float(e.nx), (float(y) + fy) / float(e.ny), (float(z) + fz) / float(e.nz));
    return __ldg(e.prob + voxel);
}

// The probability of the voxel that texture-space point uvw falls in, under the grid's address
// mode (Grid_emission::emission_pdf without its factor, volumetric_grid.cpp:104-108).
__device__ __forceinline__ float emission_prob(Emission_dist_gpu const& e, V3 uvw) {
    bool const  repeat = e.repeat != 0;
    float const u      = repeat ? uvw.x - floorf(uvw.x) : __saturatef(uvw.x);
    float const v      = repeat ? uvw.y - floorf(uvw.y) : __saturatef(uvw.y);
    float const w      = repeat ? uvw.z - floorf(uvw.z) : __saturatef(uvw.z);
    int const   x      = min(int(u * float(e.nx)), e.nx - 1);
    int const   y      = min(int(v * float(e.ny)), e.ny - 1);
    int const   z      = min(int(w * float(e.nz)), e.nz - 1);
    return __ldg(e.prob + (size_t(z) * e.ny + y) * e.nx + x);
}

// Next-event sample of an emitting medium's light: a point inside the cube -- uniform for a
// homogeneous medium (Cube::sample_volume, cube.cpp:134-151), from the emission distribution for
// a density grid (volume_image_sample, light.cpp:112-134, and Cube::sample_volume with uvw,
// cube.cpp:177-190) -- with pdf distance^2 / volume (times the voxel's probability times the
// grid's factor); its radiance is the medium's absorption times emission
// (Homogeneous::evaluate_radiance), or for a grid the nearest density times a_norm times the
// emission (Grid_emission::evaluate_radiance with Filter::Nearest, Pathtracer_MIS::evaluate_light).
__device__ void color_coefficients(Medium_gpu const& g, V3 uvw, bool nearest, float anisotropy, V3& mu_a,
                                   V3& mu_s);

__device__ bool sample_volume_light(Scene_gpu const& s, uint32_t index, V3 ps, V3 n, bool total_sphere,
                                    float pick_pdf, float r1, float r2, float r3, Light_sample& ls) {
    Volume_light_gpu const  vl   = s.volume_lights[index];
    shading::Material const lmat = s.materials[vl.material];
    V3                      uvw  = v3(r1, r2, r3);
    float                   pdf  = 1.f;
    V3                      rad  = lmat.mu_a * lmat.emission;
    if (vl.dist != 0) {
        uint32_t    voxel;
        float const prob = sample_emission(s.emission_dists[vl.dist - 1], r1, r2, r3, voxel, uvw);
        if (!(prob > 0.f)) {
            return false;
        }
        pdf = prob * vl.pdf_factor;
        Medium_gpu const& g = s.media[vl.medium];
        V3 const    e = g.temperature ? blackbody_emission(g.blackbody, __ldg(g.temperature + voxel)) : lmat.emission;
        float const d = __ldg(g.density + voxel) * (g.scale ? __ldg(g.scale + voxel) : 1.f);
        rad           = (d * vl.a_norm) * e;
    } else if (vl.color != 0) {
        // a colour grid's Volume light: its absorption at the point, nearest voxel
        // (Grid_color::evaluate_radiance with Filter::Nearest, volumetric_grid.cpp:336-343)
        V3 ma, ms;
        color_coefficients(s.media[vl.medium], uvw, true, lmat.g, ma, ms);
        rad = ma * lmat.emission;
    }
    V3 const    o    = v3(2.f * uvw.x - 1.f, 2.f * uvw.y - 1.f, 2.f * uvw.z - 1.f);
    V3 const    wp   = v3(vl.m0.x * o.x + vl.m0.y * o.y + vl.m0.z * o.z + vl.m0.w,
                          vl.m1.x * o.x + vl.m1.y * o.y + vl.m1.z * o.z + vl.m1.w,
                          vl.m2.x * o.x + vl.m2.y * o.y + vl.m2.z * o.z + vl.m2.w);
    V3 const    axis = wp - ps;
    float const d2   = shading::dot(axis, axis);
    float const d    = sqrtf(d2);
    V3 const    dir  = (1.f / d) * axis;
    if (!(d > 0.f) || (!total_sphere && !(shading::dot(dir, n) > 0.f))) {
        return false;
    }
    ls.dir      = dir;
    ls.dist     = d;
    ls.pdf      = pick_pdf * (d2 / vl.volume) * pdf;
    ls.radiance = rad;
    return true;
}

__device__ __forceinline__ bool sample_light(Scene_gpu const& s, V3 ps, V3 n, bool total_sphere,
                                             Light_pick pk, float r1, float r2, Rng& rng, Light_sample& ls) {
    if (pk.light == Env_pick) {
        // The environment: uniform directions over the hemisphere of n, or over the sphere at a
        // medium vertex (Infinite_sphere::sample, infinite_sphere.cpp:68-101).
        float const z   = total_sphere ? 1.f - 2.f * r1 : r1;
        float const rad = sqrtf(fmaxf(0.f, 1.f - z * z));
        float       sp, cp;
        sincosf(2.f * shading::Pi * r2, &sp, &cp);
        shading::Frame const f = shading::make_frame(n);
        ls.dir      = (rad * cp) * f.t + (rad * sp) * f.b + z * f.n;
        ls.dist     = Ray_max_t;
        ls.pdf      = pk.pdf * (total_sphere ? 1.f / (4.f * shading::Pi) : 1.f / (2.f * shading::Pi));
        ls.radiance = v3(s.env.x, s.env.y, s.env.z);
        return true;
    }
    if (!(pk.pdf > 0.f)) {
        return false;
    }
    uint32_t const l       = pk.light;
    float4 const   la      = s.light_tris[3 * l + 0];
    if (la.w < 0.f) {
        return sample_volume_light(s, uint32_t(-1.f - la.w), ps, n, total_sphere, pk.pdf, r1, r2, rng.uniform(),
                                   ls);
    }
    float4 const   le1     = s.light_tris[3 * l + 1];
    float4 const   le2     = s.light_tris[3 * l + 2];
    uint32_t const lmat_id = __float_as_uint(le2.w);  // the emitter's material
    float const    sq      = sqrtf(r1);
    V3 const       q       = f3v(la) + (sq * (1.f - r2)) * f3v(le1) + (sq * r2) * f3v(le2);
    V3             ln      = shading::normalize(shading::cross(f3v(le1), f3v(le2)));
    shading::Material const lmat = s.materials[lmat_id];
    if (lmat.two_sided && shading::dot(ln, q - ps) > 0.f) {
        ln = -ln;
    }
    V3 const    axis = offset_ray(q, ln) - ps;
    float const d2   = shading::dot(axis, axis);
    float const d    = sqrtf(d2);
    V3 const    dir  = (1.f / d) * axis;
    float const cl   = -shading::dot(ln, dir);
    if (!(cl >= shading::Dot_min)) {
        return false;
    }
    ls.dir      = dir;
    ls.dist     = d;
    ls.pdf      = pk.pdf * d2 / (cl * la.w);
    ls.radiance = lmat.emission;
    return true;
}

// Collisions one tracking segment may take (the reference loops until the segment ends,
// tracking.cpp:286-349,473-540).  A segment that reaches the cap -- in practice only one of
// optical thickness in the tens of thousands -- ends with the weight built up so far and is
// counted (capped, Stats::tracking_capped), so that a render can show it never happened.
constexpr int Max_tracking_steps = 1 << 16;

// Homogeneous-medium tracking over [t, d] with spectral MIS (Tracking::tracking for a
// homogeneous medium, tracking.cpp:425-470): returns true on a scattering event at t_out;
// lw receives the path weight either way.
__device__ __forceinline__ bool track_homogeneous(shading::Material const& m, float t, float d,
                                                  Rng& rng, float& t_out, V3& lw, uint32_t* capped) {
    V3 const    mu_t = m.mu_a + m.mu_s;
    float const mt   = shading::max_component(mu_t);
    lw               = v3(1.f, 1.f, 1.f);
    if (!(mt > 1e-10f)) {
        return false;
    }
    float const imt  = 1.f / mt;
    V3 const    mu_n = v3(mt - mu_t.x, mt - mu_t.y, mt - mu_t.z);
    for (int step = 0; step < Max_tracking_steps; ++step) {
        float const r0 = rng.uniform();
        t -= logf(1.f - r0) * imt;
        if (t > d) {
            return false;
        }
        float const ms = ((m.mu_s.x * lw.x) + (m.mu_s.y * lw.y) + (m.mu_s.z * lw.z)) * (1.f / 3.f);
        float const mn = ((mu_n.x * lw.x) + (mu_n.y * lw.y) + (mu_n.z * lw.z)) * (1.f / 3.f);
        float const mc = ms + mn;
        if (mc < 1e-10f) {
            return false;
        }
        float const ps = ms / mc;
        float const pn = mn / mc;
        float const r1 = rng.uniform();
        if ((r1 <= 1.f - pn) & (ps > 0.f)) {
            lw    = lw * ((1.f / (mt * ps)) * m.mu_s);
            t_out = t;
            return true;
        }
        lw = lw * ((1.f / (mt * pn)) * mu_n);
    }
    atomicAdd(capped, 1u);
    return false;
}

// Tracking in an emissive homogeneous medium (Tracking::tracking with emission,
// tracking.cpp:473-540): absorption is sampled as an event beside scattering and null
// collisions, each with probability proportional to its coefficient times the path weight;
// returns 2 on absorption (li the emitted radiance, lw zero), 1 on scattering at t_out, 0 when
// the segment is passed.
__device__ __forceinline__ int track_homogeneous_emissive(shading::Material const& m, float t, float d,
                                                          Rng& rng, float& t_out, V3& lw, V3& li,
                                                          uint32_t* capped) {
    V3 const    mu_t = m.mu_a + m.mu_s;
    float const mt   = shading::max_component(mu_t);
    lw               = v3(1.f, 1.f, 1.f);
    li               = v3(0.f, 0.f, 0.f);
    if (!(mt > 1e-10f)) {
        return 0;
    }
    float const imt  = 1.f / mt;
    V3 const    mu_n = v3(mt - mu_t.x, mt - mu_t.y, mt - mu_t.z);
    for (int step = 0; step < Max_tracking_steps; ++step) {
        float const r0 = rng.uniform();
        t -= logf(1.f - r0) * imt;
        if (t > d) {
            return 0;
        }
        float const ma = ((m.mu_a.x * lw.x) + (m.mu_a.y * lw.y) + (m.mu_a.z * lw.z)) * (1.f / 3.f);
        float const ms = ((m.mu_s.x * lw.x) + (m.mu_s.y * lw.y) + (m.mu_s.z * lw.z)) * (1.f / 3.f);
        float const mn = ((mu_n.x * lw.x) + (mu_n.y * lw.y) + (mu_n.z * lw.z)) * (1.f / 3.f);
        float const mc = ma + ms + mn;
        if (mc < 1e-10f) {
            return 0;
        }
        float const c  = 1.f / mc;
        float const pa = ma * c;
        float const ps = ms * c;
        float const pn = mn * c;
        float const r1 = rng.uniform();
        if (r1 < pa) {
            li    = lw * ((1.f / (mt * pa)) * m.mu_a) * m.emission;
            lw    = v3(0.f, 0.f, 0.f);
            t_out = t;
            return 2;
        }
        if ((r1 <= 1.f - pn) & (ps > 0.f)) {
            lw    = lw * ((1.f / (mt * ps)) * m.mu_s);
            t_out = t;
            return 1;
        }
        lw = lw * ((1.f / (mt * pn)) * mu_n);
    }
    atomicAdd(capped, 1u);
    return 0;
}

// ---- heterogeneous media: density grids (Grid material, volumetric_grid.cpp) ----
// Majorants: the grid is cut into cells of Cell_dim^3 voxels; each cell stores the minimum and
// maximum density over the voxels that trilinear filtering inside it can read (the cell plus
// one voxel on every side), as the reference's Gridtree leaves do
// (volumetric_octree_builder.cpp:105-207).  The reference refines 32^3 cells by an octree to
// 8^3 leaves; here the cells are uniformly 8^3 and a 3-D DDA walks them.  Any majorant that
// bounds the density gives the same expected result.
constexpr int   Cell_log2 = 3;
constexpr float Min_mt    = 1e-10f;  // Tracking::Min_mt, tracking.hpp:70

__device__ __forceinline__ V3 to_texture(Medium_gpu const& g, V3 p) {
    return v3(g.m0.x * p.x + g.m0.y * p.y + g.m0.z * p.z + g.m0.w,
              g.m1.x * p.x + g.m1.y * p.y + g.m1.z * p.z + g.m1.w,
              g.m2.x * p.x + g.m2.y * p.y + g.m2.z * p.z + g.m2.w);
}

__device__ __forceinline__ V3 to_texture_dir(Medium_gpu const& g, V3 d) {
    return v3(g.m0.x * d.x + g.m0.y * d.y + g.m0.z * d.z, g.m1.x * d.x + g.m1.y * d.y + g.m1.z * d.z,
              g.m2.x * d.x + g.m2.y * d.y + g.m2.z * d.z);
}

// Address modes (image/texture/address_mode.hpp): clamp saturates, repeat wraps.
__device__ __forceinline__ float address(float x, bool repeat) {
    return repeat ? x - floorf(x) : __saturatef(x);
}

__device__ __forceinline__ int lower_bound(int v, int max, bool repeat) {
    return v < 0 ? (repeat ? max : 0) : v;
}

__device__ __forceinline__ int increment(int v, int max, bool repeat) {
    return v >= max ? (repeat ? 0 : max) : v + 1;
}

// Texture filtering by depth (Pathtracer_MIS::integrate, pathtracer_mis.cpp:121, and
// Sampler_cache::sampler_3D / sampler_2D, sampler_cache.cpp:40-64): a vertex of depth 0 or 1
// samples its textures with their own filter, a deeper one with the nearest texel (keeping the
// address mode); the segment after a vertex and its shadow rays track density grids with the
// vertex's filter.  A path's depth after a bounce is the depth of the vertex it left plus one.
__device__ __forceinline__ bool nearest_at_vertex(uint32_t depth) {
    return depth >= 2;
}
__device__ __forceinline__ bool nearest_after_bounce(uint32_t depth) {
    return depth >= 3;
}

// A value of the grid's voxels at texture-space point uvw: Linear_3D::sample_1
// (texture_sampler.cpp:175-188, map :256-283) or Nearest_3D (:124-172), the latter also where
// `nearest` overrides the filter.
__device__ float sample_voxels(Medium_gpu const& g, float const* __restrict__ voxels, V3 uvw, bool nearest) {
    bool const  repeat = g.flags & 2u;
    float const u      = address(uvw.x, repeat);
    float const v      = address(uvw.y, repeat);
    float const w      = address(uvw.z, repeat);
    if ((g.flags & 1u) || nearest) {
        int const x = min(int(u * float(g.nx)), g.nx - 1);
        int const y = min(int(v * float(g.ny)), g.ny - 1);
        int const z = min(int(w * float(g.nz)), g.nz - 1);
        return __ldg(voxels + (size_t(z) * g.ny + y) * g.nx + x);
    }
    float const fu = u * float(g.nx) - 0.5f;
    float const fv = v * float(g.ny) - 0.5f;
    float const fw = w * float(g.nz) - 0.5f;
    float const lu = floorf(fu);
    float const lv = floorf(fv);
    float const lw = floorf(fw);
    int const   x  = int(lu);
    int const   y  = int(lv);
    int const   z  = int(lw);
    int const   x0 = lower_bound(x, g.nx - 1, repeat);
    int const   y0 = lower_bound(y, g.ny - 1, repeat);
    int const   z0 = lower_bound(z, g.nz - 1, repeat);
    int const   x1 = increment(x, g.nx - 1, repeat);
    int const   y1 = increment(y, g.ny - 1, repeat);
    int const   z1 = increment(z, g.nz - 1, repeat);
    float const s  = fu - lu;
    float const t  = fv - lv;
    float const r  = fw - lw;
    size_t const p00 = (size_t(z0) * g.ny + y0) * g.nx;
    size_t const p01 = (size_t(z0) * g.ny + y1) * g.nx;
    size_t const p10 = (size_t(z1) * g.ny + y0) * g.nx;
    size_t const p11 = (size_t(z1) * g.ny + y1) * g.nx;
    float const c0 = __ldg(voxels + p00 + x0);
    float const c1 = __ldg(voxels + p00 + x1);
    float const c2 = __ldg(voxels + p01 + x0);
    float const c3 = __ldg(voxels + p01 + x1);
    float const c4 = __ldg(voxels + p10 + x0);
    float const c5 = __ldg(voxels + p10 + x1);
    float const c6 = __ldg(voxels + p11 + x0);
    float const c7 = __ldg(voxels + p11 + x1);
    float const b0 = (1.f - t) * ((1.f - s) * c0 + s * c1) + t * ((1.f - s) * c2 + s * c3);
    float const b1 = (1.f - t) * ((1.f - s) * c4 + s * c5) + t * ((1.f - s) * c6 + s * c7);
    return (1.f - r) * b0 + r * b1;
}

__device__ __forceinline__ float sample_density(Medium_gpu const& g, V3 uvw, bool nearest = false) {
    return sample_voxels(g, g.density, uvw, nearest);
}

// A colour grid's coefficients at uvw (Grid_color::collision_coefficients,
// volumetric_grid.cpp:345-352): alpha x attenuation(rgb, rgb, distance, anisotropy).
__device__ void color_coefficients(Medium_gpu const& g, V3 uvw, bool nearest, float anisotropy, V3& mu_a,
                                   V3& mu_s) {
    float const alpha = sample_voxels(g, g.density, uvw, nearest);
    V3 const    c     = v3(sample_voxels(g, g.rgb[0], uvw, nearest), sample_voxels(g, g.rgb[1], uvw, nearest),
                           sample_voxels(g, g.rgb[2], uvw, nearest));
    shading::attenuation(c, c, g.color_distance, anisotropy, mu_a, mu_s);
    mu_a = alpha * mu_a;
    mu_s = alpha * mu_s;
}

// Coefficients of a grid medium at uvw: density x the material's (mu_s already scaled by the
// similarity relation), or a colour grid's with its scattering scaled by srs.
__device__ __forceinline__ void grid_coefficients(Medium_gpu const& g, shading::Material const& m, V3 mu_s,
                                                  float srs, V3 uvw, bool nearest, V3& ma, V3& ms) {
    if (g.rgb[0]) {
        color_coefficients(g, uvw, nearest, m.g, ma, ms);
        ms = srs * ms;
    } else {
        float const den = sample_density(g, uvw, nearest);
        ma              = den * m.mu_a;
        ms              = den * mu_s;
    }
}

// Majorant of the total coefficient per unit density (the majorant cells hold the density's
// maximum): the material's, or a colour grid's bound over every colour.
__device__ __forceinline__ float grid_majorant(Medium_gpu const& g, shading::Material const& m, V3 mu_s, float srs) {
    return g.rgb[0] ? g.color_maj * fmaxf(srs, 1.f) : shading::max_component(m.mu_a) + shading::max_component(mu_s);
}

// A material texture at uv (Nearest_2D / Linear_2D, texture_sampler.cpp:14-121): uv scaled,
// wrapped or clamped, then the texel it falls in, or the bilinear blend of the four texels
// around it (texel centres at half-integer positions); nearest overrides the filter.
__device__ float4 sample_texture(Texture_gpu const& t, float2 uv, bool nearest = false) {
    bool const  repeat = !(t.flags & 2u);
    float const u      = address(uv.x * t.su, repeat);
    float const v      = address(uv.y * t.sv, repeat);
    if ((t.flags & 1u) || nearest) {
        int const x = min(int(u * float(t.w)), t.w - 1);
        int const y = min(int(v * float(t.h)), t.h - 1);
        return __ldg(t.texels + size_t(y) * t.w + x);
    }
    float const fu = u * float(t.w) - 0.5f;
    float const fv = v * float(t.h) - 0.5f;
    float const x0 = floorf(fu);
    float const y0 = floorf(fv);
    int const   x  = int(x0);
    int const   y  = int(y0);
    int const   xa = lower_bound(x, t.w - 1, repeat);
    int const   ya = lower_bound(y, t.h - 1, repeat);
    int const   xb = increment(x, t.w - 1, repeat);
    int const   yb = increment(y, t.h - 1, repeat);
    float const a  = fu - x0;
    float const b  = fv - y0;
    float4 const c00 = __ldg(t.texels + size_t(ya) * t.w + xa);
    float4 const c10 = __ldg(t.texels + size_t(ya) * t.w + xb);
    float4 const c01 = __ldg(t.texels + size_t(yb) * t.w + xa);
    float4 const c11 = __ldg(t.texels + size_t(yb) * t.w + xb);
    float const  w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
    return make_float4(w00 * c00.x + w10 * c10.x + w01 * c01.x + w11 * c11.x,
                       w00 * c00.y + w10 * c10.y + w01 * c01.y + w11 * c11.y,
                       w00 * c00.z + w10 * c10.z + w01 * c01.z + w11 * c11.z, 0.f);
}

// A Substitute material's parameters at a hit with texture coordinates uv
// (Material_base::set_sample, substitute_base_material.inl:36-96): the colour map replaces the
// colour; the surface map gives the roughness (mapped to [Min_roughness, 1], ggx.inl:47-49) and,
// with two channels, the metallic value; albedo and F0 follow from them.
__device__ void apply_texture_maps(Scene_gpu const& s, shading::Material& m, float2 uv, bool nearest) {
    V3    color    = m.color;
    float metallic = m.metallic;
    if (m.color_map) {
        float4 const c = sample_texture(s.textures[m.color_map - 1], uv, nearest);
        color          = v3(c.x, c.y, c.z);
    }
    if (m.surface_map) {
        float4 const c = sample_texture(s.textures[m.surface_map - 1], uv, nearest);
        float const  r = c.x * (1.f - shading::Min_roughness) + shading::Min_roughness;
        m.alpha        = r * r;
        if (m.surface_channels >= 2) {
            metallic = c.y;
        }
    }
    m.metallic = metallic;
    m.albedo   = (1.f - metallic) * color;
    m.f0       = v3(m.f0d + metallic * (color.x - m.f0d), m.f0d + metallic * (color.y - m.f0d),
                    m.f0d + metallic * (color.z - m.f0d));
}

// Walks the majorant cells that the texture-space ray o + t d crosses for t in [t0, t1],
// clipped to the grid's unit cube (outside it the medium is empty, as outside the reference's
// Gridtree, volumetric_octree.cpp:64-75).  Calls visit(cell (min, max) density, ta, tb) for
// each cell segment in order until visit returns true; returns whether it did.
template <typename Visit>
__device__ bool walk_cells(Medium_gpu const& g, V3 o, V3 d, float t0, float t1, Visit&& visit) {
    float const tiny = 1e-30f;
    V3 const    inv  = v3(1.f / (fabsf(d.x) < tiny ? copysignf(tiny, d.x) : d.x),
                          1.f / (fabsf(d.y) < tiny ? copysignf(tiny, d.y) : d.y),
                          1.f / (fabsf(d.z) < tiny ? copysignf(tiny, d.z) : d.z));
    float lo = t0;
    float hi = t1;
    {
        float const ax = -o.x * inv.x, bx = (1.f - o.x) * inv.x;
        float const ay = -o.y * inv.y, by = (1.f - o.y) * inv.y;
        float const az = -o.z * inv.z, bz = (1.f - o.z) * inv.z;
        lo = fmaxf(lo, fmaxf(fminf(ax, bx), fmaxf(fminf(ay, by), fminf(az, bz))));
        hi = fminf(hi, fminf(fmaxf(ax, bx), fminf(fmaxf(ay, by), fmaxf(az, bz))));
    }
    if (!(lo < hi)) {
        return false;
    }
    // cells per texture-space unit along each axis
    float const sx = float(g.nx) * (1.f / float(1 << Cell_log2));
    float const sy = float(g.ny) * (1.f / float(1 << Cell_log2));
    float const sz = float(g.nz) * (1.f / float(1 << Cell_log2));
    // Starting cell from the entry point.  Should rounding put it in the neighbour behind a
    // cell face, that cell's exit distance is <= lo: it is skipped (te > t fails) and the walk
    // steps on.
    int ix = min(max(int(floorf((o.x + lo * d.x) * sx)), 0), g.cx - 1);
    int iy = min(max(int(floorf((o.y + lo * d.y) * sy)), 0), g.cy - 1);
    int iz = min(max(int(floorf((o.z + lo * d.z) * sz)), 0), g.cz - 1);
    int const   step_x = d.x > 0.f ? 1 : -1;
    int const   step_y = d.y > 0.f ? 1 : -1;
    int const   step_z = d.z > 0.f ? 1 : -1;
    float       nx_t   = (float(ix + (step_x > 0)) / sx - o.x) * inv.x;
    float       ny_t   = (float(iy + (step_y > 0)) / sy - o.y) * inv.y;
    float       nz_t   = (float(iz + (step_z > 0)) / sz - o.z) * inv.z;
    float const dx_t   = fabsf(inv.x) / sx;
    float const dy_t   = fabsf(inv.y) / sy;
    float const dz_t   = fabsf(inv.z) / sz;
    float       t      = lo;
    int const   max_steps = g.cx + g.cy + g.cz + 3;
    for (int k = 0; k < max_steps; ++k) {
        float const  te   = fminf(fminf(nx_t, ny_t), fminf(nz_t, hi));
        float2 const cell = __ldg(g.cells + (size_t(iz) * g.cy + iy) * g.cx + ix);
        if (te > t && visit(cell, t, te)) {
            return true;
        }
        if (te >= hi) {
            break;
        }
        t = fmaxf(t, te);
        if (nx_t <= ny_t && nx_t <= nz_t) {
            ix += step_x;
            nx_t += dx_t;
            if (ix < 0 || ix >= g.cx) {
                break;
            }
        } else if (ny_t <= nz_t) {
            iy += step_y;
            ny_t += dy_t;
            if (iy < 0 || iy >= g.cy) {
                break;
            }
        } else {
            iz += step_z;
            nz_t += dz_t;
            if (iz < 0 || iz >= g.cz) {
                break;
            }
        }
    }
    return false;
}


// Delta tracking with spectral MIS through a density grid over the world ray (ro, rd) for t in
// [t0, t1] (Tracking_multi::integrate heterogeneous branch, tracking_multi.cpp:98-164, with
// Tracking::tracking over a majorant cell, tracking.cpp:286-349).  srs scales the scattering
// coefficient (similarity relation); nearest overrides the grid's filter.  Returns true on a
// scattering event at t_out; lw receives the path weight either way.
__device__ bool track_grid(Medium_gpu const& g, shading::Material const& m, float srs, V3 ro,
                           V3 rd, float t0, float t1, bool nearest, Rng& rng, float& t_out, V3& lw,
                           uint32_t* capped) {
    V3 const    o     = to_texture(g, ro);
    V3 const    d     = to_texture_dir(g, rd);
    V3 const    mu_s  = srs * m.mu_s;
    float const maj_t = grid_majorant(g, m, mu_s, srs);
    lw                = v3(1.f, 1.f, 1.f);
    int  steps        = 0;
    bool scattered    = false;
    walk_cells(g, o, d, t0, t1, [&](float2 cell, float ta, float tb) {
        float const mt = cell.y * maj_t;
        if (mt < Min_mt) {
            return false;
        }
        float const imt = 1.f / mt;
        for (float t = ta; steps < Max_tracking_steps; ++steps) {
            t -= logf(1.f - rng.uniform()) * imt;
            if (t > tb) {
                return false;
            }
            V3 ma, ms3;
            grid_coefficients(g, m, mu_s, srs, o + t * d, nearest, ma, ms3);
            V3 const    mu_n = v3(mt - (ma.x + ms3.x), mt - (ma.y + ms3.y), mt - (ma.z + ms3.z));
            float const ms   = ((ms3.x * lw.x) + (ms3.y * lw.y) + (ms3.z * lw.z)) * (1.f / 3.f);
            float const mn   = ((mu_n.x * lw.x) + (mu_n.y * lw.y) + (mu_n.z * lw.z)) * (1.f / 3.f);
            float const sum  = ms + mn;
            if (!(sum > 0.f)) {
                lw = v3(0.f, 0.f, 0.f);
                return true;
            }
            float const ps = ms / sum;
            float const pn = mn / sum;
            if ((rng.uniform() <= 1.f - pn) & (ps > 0.f)) {
                lw        = lw * ((1.f / (mt * ps)) * ms3);
                t_out     = t;
                scattered = true;
                return true;
            }
            lw = lw * ((1.f / (mt * pn)) * mu_n);
        }
        return true;
    });
    if (steps >= Max_tracking_steps) {
        atomicAdd(capped, 1u);
    }
    return scattered;
}

// Tracking through an emissive density grid (Grid_emission, volumetric_grid.cpp:110-127, with
// the emissive Tracking::tracking over a majorant cell, tracking.cpp:351-423): absorption is an
// event beside scattering and null collisions, each chosen in proportion to its coefficient
// times the path weight; the absorbed path carries the emission (constant over the grid; the
// density scales the absorption coefficient).  Returns 2 on absorption at t_out (li the
// emitted radiance, lw zero), 1 on scattering at t_out, 0 when the segment is passed.
__device__ int track_grid_emissive(Medium_gpu const& g, shading::Material const& m, float srs, V3 ro, V3 rd,
                                   float t0, float t1, bool nearest, Rng& rng, float& t_out, V3& lw, V3& li,
                                   uint32_t* capped) {
    V3 const    o     = to_texture(g, ro);
    V3 const    d     = to_texture_dir(g, rd);
    V3 const    mu_s  = srs * m.mu_s;
    float const maj_t = grid_majorant(g, m, mu_s, srs);
    lw                = v3(1.f, 1.f, 1.f);
    li                = v3(0.f, 0.f, 0.f);
    int steps         = 0;
    int event         = 0;
    walk_cells(g, o, d, t0, t1, [&](float2 cell, float ta, float tb) {
        float const mt = cell.y * maj_t;
        if (mt < Min_mt) {
            return false;
        }
        float const imt = 1.f / mt;
        for (float t = ta; steps < Max_tracking_steps; ++steps) {
            t -= logf(1.f - rng.uniform()) * imt;
            if (t > tb) {
                return false;
            }
            V3 ma3, ms3;
            grid_coefficients(g, m, mu_s, srs, o + t * d, nearest, ma3, ms3);
            V3 const    mu_n = v3(mt - (ma3.x + ms3.x), mt - (ma3.y + ms3.y), mt - (ma3.z + ms3.z));
            float const ma   = ((ma3.x * lw.x) + (ma3.y * lw.y) + (ma3.z * lw.z)) * (1.f / 3.f);
            float const ms   = ((ms3.x * lw.x) + (ms3.y * lw.y) + (ms3.z * lw.z)) * (1.f / 3.f);
            float const mn   = ((mu_n.x * lw.x) + (mu_n.y * lw.y) + (mu_n.z * lw.z)) * (1.f / 3.f);
            float const sum  = ma + ms + mn;
            if (!(sum > 0.f)) {
                lw = v3(0.f, 0.f, 0.f);
                return true;
            }
            float const c  = 1.f / sum;
            float const pa = ma * c;
            float const ps = ms * c;
            float const pn = mn * c;
            float const r1 = rng.uniform();
            if (r1 < pa) {
                V3 e = g.temperature ? blackbody_emission(g.blackbody, sample_voxels(g, g.temperature, o + t * d, nearest))
                                     : m.emission;
                if (g.scale) {
                    e = sample_voxels(g, g.scale, o + t * d, nearest) * e;
                }
                li    = lw * ((1.f / (mt * pa)) * ma3) * e;
                lw    = v3(0.f, 0.f, 0.f);
                t_out = t;
                event = 2;
                return true;
            }
            if ((r1 <= 1.f - pn) & (ps > 0.f)) {
                lw    = lw * ((1.f / (mt * ps)) * ms3);
                t_out = t;
                event = 1;
                return true;
            }
            lw = lw * ((1.f / (mt * pn)) * mu_n);
        }
        return true;
    });
    if (steps >= Max_tracking_steps) {
        atomicAdd(capped, 1u);
    }
    return event;
}

__device__ __forceinline__ bool all_below_abort(V3 w) {
    return w.x < Abort_epsilon && w.y < Abort_epsilon && w.z < Abort_epsilon;
}

// Transmittance of a density grid along the world ray for t in [t0, t1]: ratio tracking per
// majorant cell, residual ratio tracking against the cell's minorant where it is positive
// (tracking_transmitted / residual_ratio_tracking_transmitted, tracking.cpp:32-140).  w is
// multiplied by the estimate; returns false when it falls below Abort_epsilon (the shadow
// ray counts as blocked, Tracking::transmittance, tracking.cpp:143-180).  nearest overrides the
// grid's filter.
__device__ bool transmit_grid(Medium_gpu const& g, shading::Material const& m, float srs, V3 ro,
                              V3 rd, float t0, float t1, bool nearest, Rng& rng, V3& w, uint32_t* capped) {
    V3 const    o     = to_texture(g, ro);
    V3 const    d     = to_texture_dir(g, rd);
    V3 const    mu_s  = srs * m.mu_s;
    float const maj_t = grid_majorant(g, m, mu_s, srs);
    // a colour grid has no minorant here: plain ratio tracking
    float const min_t = g.rgb[0] ? 0.f : shading::min_component(m.mu_a) + shading::min_component(mu_s);
    int  steps        = 0;
    bool blocked      = false;
    walk_cells(g, o, d, t0, t1, [&](float2 cell, float ta, float tb) {
        float const mt = cell.y * maj_t;
        if (mt < Min_mt) {
            return false;
        }
        // Control medium: the cell's minorant mu_t, whose transmittance is analytic; ratio
        // tracking then samples only the residual (plain ratio tracking when it is 0).
        float const cm = fmaxf(cell.x * min_t, 0.f);
        if (cm > 0.f) {
            w = expf(-(tb - ta) * cm) * w;
            if (all_below_abort(w)) {
                blocked = true;
                return true;
            }
        }
        float const mr = mt - cm;
        if (mr < Min_mt) {
            return false;
        }
        float const imr = 1.f / mr;
        for (float t = ta; steps < Max_tracking_steps; ++steps) {
            t -= logf(1.f - rng.uniform()) * imr;
            if (t > tb) {
                return false;
            }
            V3 mt3;
            if (g.rgb[0]) {
                V3 ma, ms;
                color_coefficients(g, o + t * d, nearest, m.g, ma, ms);
                mt3 = ma + srs * ms;
            } else {
                mt3 = sample_density(g, o + t * d, nearest) * (m.mu_a + mu_s);
            }
            w = v3(w.x * ((mr - (mt3.x - cm)) * imr), w.y * ((mr - (mt3.y - cm)) * imr),
                   w.z * ((mr - (mt3.z - cm)) * imr));
            if (all_below_abort(w)) {
                blocked = true;
                return true;
            }
        }
        return false;
    });
    if (steps >= Max_tracking_steps) {
        atomicAdd(capped, 1u);
    }
    return !blocked;
}

// Light samples at a vertex of the given depth: two (the environment, and an emitter) where
// the selection is split and both kinds of light exist, else one (0 without lights).
// Whether light selection at a vertex of this depth splits (Pathtracer_MIS::splitting).
__device__ __forceinline__ bool splits_at(Scene_gpu const& s, uint32_t depth) {
    return depth < s.split_bounces;
}

__device__ __forceinline__ void store_shadow(Paths const& p, uint32_t path, bool second, V3 o,
                                             Light_sample const& ls, V3 contrib, uint32_t depth) {
    float4 const ro = make_float4(o.x, o.y, o.z, 0.f);
    float4 const rd = make_float4(ls.dir.x, ls.dir.y, ls.dir.z, ls.dist);
    float4 const c  = make_float4(contrib.x, contrib.y, contrib.z, float(depth));
    if (second) {
        p.sh2_o[path] = ro;
        p.sh2_d[path] = rd;
        p.sh2_L[path] = c;
    } else {
        p.sh_o[path] = ro;
        p.sh_d[path] = rd;
        p.sh_L[path] = c;
    }
}

// The wave's queues and counters k_shade appends to.
struct Shade_out {
    uint32_t* q_out;          // extension queue of the next vertex
    uint32_t* count_out;
    uint32_t* sq;             // shadow queue
    uint32_t* count_shadow;
    uint32_t* count_picks;    // picks of split selections
    uint32_t* count_records;  // split records
};

// Next-event estimation at a vertex (sample_lights / evaluate_light, pathtracer_mis.cpp:281-347):
// the lights select_lights chooses with the random number `select`, a sample on each (the
// pixel's golden ratio dimension of that light at the first vertices, else the path's random
// stream), and each sample's contribution eval(ls).  The environment of a split selection (its
// first light) takes the path's second shadow slot; a single other light the first slot;
// several emitters get a split record and a pick each, their contributions summed by
// k_pick_sum after the shadow rays.  shadow / shadow2: the slots hold rays.
template <class Eval>
__device__ __forceinline__ void next_event(Scene_gpu const& s, Paths const& p, Wave const& wave,
                                           Shade_out const& out, uint32_t path, V3 ps, V3 n,
                                           bool total_sphere, uint32_t depth, float select, Rng& rng,
                                           bool golden, uint32_t gpixel, uint32_t gsample, Eval const& eval,
                                           bool& shadow, bool& shadow2) {
    // One walk counts the selection and keeps its first two lights; a split selection of more
    // (rare) walks again for each further light.
    bool const split  = splits_at(s, depth);
    Light_pick first0 = {0u, 0.f}, first1 = {0u, 0.f};
    uint32_t const m  = walk_lights(s, ps, n, total_sphere, select, split, [&](uint32_t k, Light_pick pk) {
        if (k == 0) {
            first0 = pk;
        } else if (k == 1) {
            first1 = pk;
        }
        return true;
    });
    auto const pick_at = [&](uint32_t k) {
        if (k < 2) {
            return k == 0 ? first0 : first1;
        }
        Light_pick got = {0u, 0.f};
        walk_lights(s, ps, n, total_sphere, select, split, [&](uint32_t i, Light_pick pk) {
            got = pk;
            return i < k;
        });
        return got;
    };
    auto const     point = [&](uint32_t l, float& r1, float& r2) {
        if (golden) {
            float2 const g = golden_2d(wave, gpixel, gsample, golden_light_2d(depth, l));
            r1             = g.x;
            r2             = g.y;
        } else {
            r1 = rng.uniform();
            r2 = rng.uniform();
        }
    };
    auto const slot = [&](uint32_t l, bool second) {
        float r1, r2;
        point(l, r1, r2);
        Light_sample ls;
        if (sample_light(s, ps, n, total_sphere, pick_at(l), r1, r2, rng, ls)) {
            V3 const c = eval(ls);
            if (shading::max_component(c) > 0.f) {
                store_shadow(p, path, second, ps, ls, c, depth);
                return true;
            }
        }
        return false;
    };
    uint32_t first = 0;
    if (m > 1 && first0.light == Env_pick) {
        shadow2 = slot(0, true);
        first   = 1;
    }
    uint32_t const count = m - first;
    if (count == 1) {
        shadow = slot(first, false);
    }
    if (count < 2) {
        return;
    }
    uint32_t const base = atomicAdd(out.count_picks, count);
    uint32_t const rec  = atomicAdd(out.count_records, 1u);
    p.split_o[rec]      = make_float4(ps.x, ps.y, ps.z, __uint_as_float(path));
    p.split_m[rec]      = make_uint4(base, count, depth, 0u);
    uint64_t valid      = 0;
    for (uint32_t k = 0; k < count; ++k) {
        float r1, r2;
        point(first + k, r1, r2);
        Light_sample ls;
        V3           c = v3(0.f, 0.f, 0.f);
        float4       d = make_float4(0.f, 0.f, 1.f, 0.f);
        if (sample_light(s, ps, n, total_sphere, pick_at(first + k), r1, r2, rng, ls)) {
            V3 const e = eval(ls);
            if (shading::max_component(e) > 0.f) {
                c = e;
                d = make_float4(ls.dir.x, ls.dir.y, ls.dir.z, ls.dist);
                valid |= 1ull << k;
            }
        }
        p.pick_d[base + k] = d;
        p.pick_c[base + k] = make_float4(c.x, c.y, c.z, __uint_as_float(rec));
    }
    if (valid != 0) {
        uint32_t q = atomicAdd(out.count_shadow, uint32_t(__popcll(valid)));
        for (uint32_t k = 0; k < count; ++k) {
            if ((valid >> k) & 1u) {
                out.sq[q++] = Pick_shadow | (base + k);
            }
        }
    }
}

// Sums each split record's picks (in pick order) into its path's L2, after the bounce's shadow
// rays have zeroed the occluded ones.
__global__ void __launch_bounds__(256)
    k_pick_sum(Paths p, uint32_t const* __restrict__ count) {
    uint32_t const num = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < num; i += gridDim.x * blockDim.x) {
        float4 const o = p.split_o[i];
        uint4 const  m = p.split_m[i];
        float        x = 0.f, y = 0.f, z = 0.f;
        for (uint32_t l = 0; l < m.y; ++l) {
            float4 const c = p.pick_c[m.x + l];
            x += c.x;
            y += c.y;
            z += c.z;
        }
        uint32_t const path = __float_as_uint(o.w);
        float4         l2   = p.L2[path];
        l2.x += x;
        l2.y += y;
        l2.z += z;
        p.L2[path] = l2;
    }
}

// ---- guide: the network's mixture for every queued surface hit (before shading) ----
// Two kernels per bounce.  k_guide_encode, one thread per queue entry, encodes the hit
// (position in the scene box, geometric normal facing the ray's origin, outgoing direction)
// into guide_in and marks the entry guided (a Substitute surface below the guided depth).
// k_guide streams those tiles through the network on the tensor cores (guide_mlp.cuh) and
// stores each entry's mixture at its queue position, where k_shade reads it.
struct Infer_smem {
    guide::Net_smem net;
    // Per tile of the pair being processed: two activation buffers (the second's first 8 KB
    // also take the tile's inputs); after the last layer the 32 KB hold its 128 output rows.
    __nv_bfloat16 act[2][2][guide::Tile * guide::Width];
    uint64_t      mbar[2];    // tensor-core completion barriers
    uint32_t      tmem_slot;  // accumulator address from tcgen05.alloc
};
static_assert(sizeof(float) * 48 * guide::Tile <= sizeof(__nv_bfloat16) * 2 * guide::Tile * guide::Width,
              "a tile's mixture rows fit its activation buffers");

// Position, geometric normal (facing -dir) and outgoing direction of a path's hit.
__device__ __forceinline__ void hit_frame(Scene_gpu const& s, Paths const& p, uint32_t path, uint32_t id,
                                          V3& pos, V3& geo_n, V3& wo) {
    World_tri const w  = world_triangle(s, hit_instance(s, p, path), id);
    float2 const    uv = p.hit_uv[path];
    pos                = (1.f - uv.x - uv.y) * w.a + uv.x * w.b + uv.y * w.c;
    geo_n              = shading::normalize(shading::cross(w.b - w.a, w.c - w.a));
    wo               = -f3v(p.ray_d[path]);
    if (shading::dot(geo_n, wo) < 0.f) {
        geo_n = -geo_n;
    }
}

__device__ __forceinline__ V3 box_coordinates(Wave const& wave, V3 pos) {
    return v3((pos.x - wave.bounds_lo.x) * wave.bounds_inv.x, (pos.y - wave.bounds_lo.y) * wave.bounds_inv.y,
              (pos.z - wave.bounds_lo.z) * wave.bounds_inv.z);
}

// One queue entry per thread: its inputs as row q % 128 of tile q / 128 (entries past the
// queue's end, up to the tile boundary, get zeros).
__global__ void __launch_bounds__(256)
    k_guide_encode(Scene_gpu s, Launch const* __restrict__ launch, Paths p, uint32_t const* __restrict__ queue,
                   uint32_t const* __restrict__ count) {
    Wave const&    wave = launch->wave;
    uint32_t const q   = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t const num = *count;
    if (q >= (num + guide::Tile - 1) / guide::Tile * guide::Tile) {
        return;
    }
    float in[guide::Inputs];
    bool  ok = false;
    if (q < num) {
        uint32_t const path  = queue[q];
        uint32_t const id    = p.hit_id[path];
        uint32_t const depth = (p.info[path] >> 8) & 0xFFu;
        if (id != gpu::Miss && depth < wave.guide_depth &&
            s.materials[world_triangle(s, hit_instance(s, p, path), id).material].type ==
                shading::Type_substitute) {
            V3 pos, geo_n, wo;
            hit_frame(s, p, path, id, pos, geo_n, wo);
            guide::encode(box_coordinates(wave, pos), geo_n, wo, in);
            ok = true;
        }
        p.guide_ok[q] = ok ? 1 : 0;
    }
    __nv_bfloat16* const tile = p.guide_in + size_t(q / guide::Tile) * guide::Tile * guide::Inputs;
    int const            r    = int(q % guide::Tile);
#pragma unroll
    for (int k = 0; k < guide::Inputs; k += 8) {
        __nv_bfloat162 h[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            h[j] = __floats2bfloat162_rn(ok ? in[k + 2 * j] : 0.f, ok ? in[k + 2 * j + 1] : 0.f);
        }
        *reinterpret_cast<uint4*>(tile + guide::tiled(r, k, guide::Inputs)) = *reinterpret_cast<uint4*>(h);
    }
}

// The last layer of one tile, by all threads: thread t takes row t % 128 and lobes 4h..4h+3
// (h = t / 128) of it -- their 16 outputs and the 8 mixture logits from the accumulator plus
// bias -- and writes them as guide::mixture does (unit mean, concentration, softmax weight),
// with the hardware exponential, into `rows` in the Mixture_floats form.
__device__ __forceinline__ void finish_mixture(float const* b, float4* rows, guide::Tmem_tile& tm) {
    if (!guide::mbar_wait(tm.mbar, tm.phase)) {
        *tm.error = 1u;
    }
    tm.phase ^= 1u;
    guide::tc_fence_after();
    int const      warp  = threadIdx.x >> 5;
    int const      r     = threadIdx.x & (guide::Tile - 1);
    int const      h     = threadIdx.x >> 7;
    uint32_t const lanes = uint32_t(32 * (warp & 3)) << 16;
    float          m[16], logit[8];
    guide::tmem_ld16(tm.tmem + lanes + uint32_t(16 * h), m);
    guide::tmem_ld8(tm.tmem + lanes + 32u, logit);
    float mx = -3.4e38f;
#pragma unroll
    for (int j = 0; j < guide::Lobes; ++j) {
        logit[j] += b[32 + j];
        mx = fmaxf(mx, logit[j]);
    }
    float sum = 0.f, mine[4];
#pragma unroll
    for (int j = 0; j < guide::Lobes; ++j) {
        float const e = __expf(logit[j] - mx);
        sum += e;
        if (j / 4 == h) {
            mine[j % 4] = e;
        }
    }
    float const inv = 1.f / sum;
    float4* const row = rows + r * (Mixture_floats / 4);
    float         norm[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int const   o  = 16 * h + 4 * j;
        float const x  = m[4 * j] + b[o];
        float const y  = m[4 * j + 1] + b[o + 1];
        float const z  = m[4 * j + 2] + b[o + 2];
        float const lk = m[4 * j + 3] + b[o + 3];
        float const l2 = x * x + y * y + z * z;
        float const s  = l2 > 1e-20f ? rsqrtf(l2) : 0.f;
        float const k  = __expf(fminf(fmaxf(lk, guide::Log_kappa_min), guide::Log_kappa_max));
        row[4 * h + j] = l2 > 1e-20f ? make_float4(s * x, s * y, s * z, k) : make_float4(0.f, 0.f, 1.f, k);
        norm[j]        = k / (2.f * 3.14159265358979f * -expm1f(-2.f * k));
        mine[j] *= inv;
    }
    row[8 + h]  = make_float4(mine[0], mine[1], mine[2], mine[3]);
    row[10 + h] = make_float4(mine[0] * norm[0], mine[1] * norm[1], mine[2] * norm[2], mine[3] * norm[3]);
}

// Persistent: each block loads the network once, then walks pairs of tiles, the two
// interleaved layer by layer so that one tile's MMAs run while the other's results are stored;
// the next pair's 16 KB of inputs are read into registers meanwhile.  The mixture rows, staged
// in shared memory, are written to guide_out (entry q at q * Mixture_floats) as contiguous
// 16-byte stores.
constexpr uint32_t Infer_tmem_columns = 2 * guide::Tmem_columns;

__global__ void __launch_bounds__(guide::Block, 2)
    k_guide(Paths p, uint32_t const* __restrict__ count, __nv_bfloat16 const* __restrict__ wbf,
            float const* __restrict__ params, uint32_t* error) {
    extern __shared__ __align__(16) unsigned char raw[];
    Infer_smem&    m     = *reinterpret_cast<Infer_smem*>(raw);
    uint32_t const num   = *count;
    uint32_t const tiles = (num + guide::Tile - 1) / guide::Tile;
    uint32_t const pairs = (tiles + 1) / 2;
    if (blockIdx.x >= pairs) {
        return;  // the whole block: no barrier is skipped by only some threads
    }
    constexpr int Tile_uint4 = guide::Tile * guide::Inputs * 2 / 16;  // 512
    static_assert(Tile_uint4 == 2 * guide::Block, "two 16-byte loads per thread per tile");
    uint4 const* const src  = reinterpret_cast<uint4 const*>(p.guide_in);
    uint4 const        zero = make_uint4(0u, 0u, 0u, 0u);
    auto const         load = [&](uint32_t tile, int half) {
        return tile < tiles ? src[size_t(tile) * Tile_uint4 + half * guide::Block + threadIdx.x] : zero;
    };
    uint4 n[4] = {load(2 * blockIdx.x, 0), load(2 * blockIdx.x, 1), load(2 * blockIdx.x + 1, 0),
                  load(2 * blockIdx.x + 1, 1)};
    guide::load_net(m.net, wbf, params);
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         guide::smem_u32(&m.tmem_slot)),
                     "r"(Infer_tmem_columns));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int t = 0; t < 2; ++t) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(guide::smem_u32(&m.mbar[t])), "r"(1));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    guide::tc_fence_before();
    __syncthreads();
    guide::tc_fence_after();
    guide::Tmem_tile tm[2] = {{m.tmem_slot, guide::smem_u32(&m.mbar[0]), 0u, error},
                              {m.tmem_slot + guide::Tmem_columns, guide::smem_u32(&m.mbar[1]), 0u, error}};
    guide::Smem_outputs const unused{nullptr};
    float const* const        b = m.net.b;
#pragma unroll 1
    for (uint32_t pair = blockIdx.x; pair < pairs; pair += gridDim.x) {
        for (int t = 0; t < 2; ++t) {
            uint4* const in = reinterpret_cast<uint4*>(m.act[t][1]);
            in[threadIdx.x]                = n[2 * t];
            in[guide::Block + threadIdx.x] = n[2 * t + 1];
        }
        uint32_t const next = pair + gridDim.x;
        if (next < pairs) {
            n[0] = load(2 * next, 0);
            n[1] = load(2 * next, 1);
            n[2] = load(2 * next + 1, 0);
            n[3] = load(2 * next + 1, 1);
        }
        guide::fence_async_smem();
        guide::tc_fence_before();
        __syncthreads();
        // layer l reads act[t][(l + 1) & 1] and writes act[t][l & 1]
        guide::issue_layer<guide::Inputs, guide::Width>(m.act[0][1], m.net.w + guide::weight_tile_offset(0), tm[0]);
        guide::issue_layer<guide::Inputs, guide::Width>(m.act[1][1], m.net.w + guide::weight_tile_offset(0), tm[1]);
#pragma unroll
        for (int l = 0; l < guide::Layers - 1; ++l) {
            __nv_bfloat16 const* w_next = m.net.w + guide::weight_tile_offset(l + 1);
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                guide::finish_layer<guide::Width, false>(b + guide::bias_slot(l), m.act[t][l & 1], unused, tm[t]);
                if (l + 1 < guide::Layers - 1) {
                    guide::issue_layer<guide::Width, guide::Width>(m.act[t][l & 1], w_next, tm[t]);
                } else {
                    guide::issue_layer<guide::Width, guide::Outputs>(m.act[t][l & 1], w_next, tm[t]);
                }
            }
        }
        // Last layer: both tiles' rows into their (now free) activation buffers, then out.
        for (int t = 0; t < 2; ++t) {
            finish_mixture(b + guide::bias_slot(guide::Layers - 1), reinterpret_cast<float4*>(m.act[t]), tm[t]);
        }
        guide::tc_fence_before();
        __syncthreads();
        for (int t = 0; t < 2; ++t) {
            uint32_t const base = (2 * pair + uint32_t(t)) * guide::Tile;
            uint32_t const rows = base < num ? min(uint32_t(guide::Tile), num - base) : 0u;
            uint4 const*   from = reinterpret_cast<uint4 const*>(m.act[t]);
            uint4* const   to   = reinterpret_cast<uint4*>(p.guide_out + size_t(base) * Mixture_floats);
            for (uint32_t i = threadIdx.x; i < rows * (Mixture_floats / 4); i += guide::Block) {
                to[i] = from[i];
            }
        }
        __syncthreads();  // the rows are read before the next pair's inputs replace them
    }
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm[0].tmem), "r"(Infer_tmem_columns));
    }
}

// ---- the guide's mixture as k_guide stores it per queue entry ----
// (Mixture_floats per entry; read through L1 by each use.)

__device__ __forceinline__ float mixture_pdf_at(float4 const* __restrict__ row, V3 w) {
    float4 const c0 = row[10], c1 = row[11];
    float const  c[guide::Lobes] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    float        q = 0.f;
#pragma unroll
    for (int j = 0; j < guide::Lobes; ++j) {
        float4 const l = row[j];
        q += c[j] * __expf(l.w * (l.x * w.x + l.y * w.y + l.z * w.z - 1.f));
    }
    return q;
}

// Samples the stored mixture with three uniform numbers: a lobe by weight, then its vMF.
__device__ __forceinline__ V3 mixture_sample_at(float4 const* __restrict__ row, float u0, float u1, float u2) {
    float4 const w0 = row[8], w1 = row[9];
    float const  w[guide::Lobes] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    int          j   = guide::Lobes - 1;
    float        acc = 0.f;
#pragma unroll
    for (int k = 0; k < guide::Lobes - 1; ++k) {
        acc += w[k];
        if (u0 < acc) {
            j = k;
            break;
        }
    }
    float4 const l = row[j];
    guide::Lobe  lobe;
    lobe.mu     = v3(l.x, l.y, l.z);
    lobe.kappa  = l.w;
    lobe.weight = 1.f;
    return guide::vmf_sample(lobe, u1, u2);
}

// Russian roulette's continuation probability (russian_roulette, integrator_helper.hpp:42-52):
// the throughput's largest component.  The reference does not clamp it to 1 -- a throughput
// above 1 then scales the path down, a bias it never meets with its BSDF sampling alone
// (f cos / pdf stays below 1), and plain MIS here mirrors it.  Guided paths, whose throughput
// f cos / (mixed pdf) can exceed 1, use the clamped, unbiased probability.
__device__ __forceinline__ float continuation_probability(Wave const& wave, V3 T) {
    float const q = shading::max_component(T);
    return wave.guiding ? fminf(q, 1.f) : q;
}

// The pdf with which next-event estimation from the previous vertex would have drawn the point
// at distance t along the ray inside an emitting medium's light (connect_light_volume,
// pathtracer_mis.cpp:382-400, with Light::pdf for Volume and Volume_image lights,
// light.cpp:352-362): the light-tree pick from that vertex times distance^2 / volume, times the
// voxel's probability and the grid's factor for a density grid.
__device__ float volume_light_pdf(Scene_gpu const& s, Paths const& p, uint32_t path, shading::Material const& m,
                                  V3 ro, V3 rd, float t, uint32_t depth) {
    uint32_t const         order = m.volume_light - 1;
    float4 const           pn    = p.prev_n[path];
    float const            pick  = light_pick_pdf(s, ro, f3v(pn), pn.w != 0.f, order, splits_at(s, depth));
    Volume_light_gpu const vl    = s.volume_lights[uint32_t(-1.f - s.light_tris[3 * order].w)];
    float                  pdf   = pick * (t * t) / vl.volume;
    if (vl.dist != 0) {
        Medium_gpu const& g   = s.media[vl.medium];
        V3 const          uvw = to_texture(g, ro + t * rd);
        pdf *= emission_prob(s.emission_dists[vl.dist - 1], uvw) * vl.pdf_factor;
    }
    return pdf;
}

// ---- shade: one path vertex ----
__global__ void __launch_bounds__(Shade_block)
    k_shade(Scene_gpu s, Launch const* __restrict__ launch, Paths p, uint32_t const* __restrict__ q_in,
            uint32_t const* __restrict__ count_in, Shade_out out) {
    Wave const&    wave = launch->wave;
    uint32_t const i   = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t const num = *count_in;

    bool     extend  = false;
    bool     shadow  = false;  // the path's first shadow slot holds a ray
    bool     shadow2 = false;  // ... its second
    uint32_t path    = 0;

    if (i < num) {
        path              = q_in[i];
        uint32_t info     = p.info[path];
        uint32_t vtx      = info & 0xFFu;
        uint32_t depth    = (info >> 8) & 0xFFu;
        bool     singular = (info >> 16) & 1u;
        uint32_t medium   = info >> 17;  // material index + 1 of the medium the path is in
        float4   T4       = p.T[path];
        V3       T        = f3v(T4);
        float    bsdf_pdf = T4.w;
        float4   L4       = p.L[path];
        V3       L        = f3v(L4);
        uint32_t const id = p.hit_id[path];
        bool     done     = false;
        if (wave.record_depth) {
            // The training record of the previous vertex learns what its continuation found:
            // the radiance gathered so far (its own light samples included) marks the start.
            uint32_t const open = p.open_record[path];
            if (open != 0xFFFFFFFFu) {
                float4 const l2 = p.L2[path];
                p.rec[size_t(open) * Record_float4 + 4] = make_float4(L.x + l2.x, L.y + l2.y, L.z + l2.z, 1.f);
                p.open_record[path] = 0xFFFFFFFFu;
            }
        }
        float4 const ro   = p.ray_o[path];
        float4 const rd   = p.ray_d[path];
        V3 const     dir_in = v3(rd.x, rd.y, rd.z);

        Rng rng;
        rng.load(p.rng[path]);

        // Inside a medium: track to the next surface (Tracking_multi::integrate,
        // tracking_multi.cpp:45-238); leaving to infinity ends the path.
        bool  scatter = false;
        float t_sc    = 0.f;
        if (id == gpu::Miss) {
            // Leaving the scene: the uniform environment (an Infinite_sphere prop).  The camera
            // sees it; continuation rays only when it is a light, weighted against its NEE pdf
            // from the previous vertex (connect_light, pathtracer_mis.cpp:349-380).
            if (medium == 0 && (vtx == 0 || s.env.w > 0.f)) {
                float w = 1.f;
                if (vtx > 0 && !singular) {
                    float4 const pn    = p.prev_n[path];
                    float const  pdf_e = (splits_at(s, depth) ? 1.f : s.env.w) *
                                         (pn.w != 0.f ? 1.f / (4.f * shading::Pi)
                                                      : 1.f / (2.f * shading::Pi));
                    w = power_heuristic(bsdf_pdf, pdf_e);
                }
                L = L + w * (T * v3(s.env.x, s.env.y, s.env.z));
            }
            done = true;
        } else if (medium != 0) {
            shading::Material const m = s.materials[medium - 1];
            V3 lw;
            bool const emissive = m.emission.x > 0.f || m.emission.y > 0.f || m.emission.z > 0.f;
            if (emissive) {
                // An emitting medium: an absorption event ends the path with the emitted
                // radiance (pathtracer_mis.cpp:214-231).  The camera segment takes all of it;
                // later segments take it only from a light, weighed against next-event
                // estimation of that light from the previous vertex (connect_light_volume,
                // pathtracer_mis.cpp:382-400).
                V3        li;
                int const ev = m.medium != 0
                                   ? track_grid_emissive(s.media[m.medium - 1], m,
                                                         shading::similarity_relation_scale(m.g, depth), f3v(ro),
                                                         dir_in, ro.w, p.hit_t[path], nearest_after_bounce(depth),
                                                         rng, t_sc, lw, li, s.tracking_capped)
                                   : track_homogeneous_emissive(m, ro.w, p.hit_t[path], rng, t_sc, lw, li,
                                                                s.tracking_capped);
                if (ev == 2 && (depth == 0 || m.volume_light != 0)) {
                    float w = 1.f;
                    if (depth > 0 && !singular && m.volume_light != shading::Volume_light_unsampled) {
                        w = power_heuristic(bsdf_pdf, volume_light_pdf(s, p, path, m, f3v(ro), dir_in, t_sc, depth));
                    }
                    L = L + w * (T * li);
                }
                scatter = ev == 1;
            } else if (m.medium != 0) {
                float const srs = shading::similarity_relation_scale(m.g, depth);
                scatter = track_grid(s.media[m.medium - 1], m, srs, f3v(ro), dir_in, ro.w, p.hit_t[path],
                                     nearest_after_bounce(depth), rng, t_sc, lw, s.tracking_capped);
            } else {
                scatter = track_homogeneous(m, ro.w, p.hit_t[path], rng, t_sc, lw, s.tracking_capped);
            }
            T = T * lw;
            if (!(lw.x >= Abort_epsilon || lw.y >= Abort_epsilon || lw.z >= Abort_epsilon)) {
                done = true;
            }
        }

        if (!done && scatter) {
            // Scattering vertex inside the medium (volumetric::Sample, HG phase function).
            if (depth >= wave.max_bounces) {
                done = true;
            } else if (depth >= wave.min_bounces) {
                float const q = continuation_probability(wave, T);
                if (rng.uniform() > q) {
                    done = true;
                } else {
                    T = (1.f / q) * T;
                }
            }
            if (!done) {
                shading::Material const m = s.materials[medium - 1];
                float const g   = shading::van_de_hulst_anisotropy(m.g, depth);
                V3 const    pos = v3(ro.x + t_sc * rd.x, ro.y + t_sc * rd.y, ro.z + t_sc * rd.z);
                V3 const    wo  = -dir_in;
                float const select = rng.uniform();
                next_event(s, p, wave, out, path, pos, v3(0.f, 0.f, 1.f), true, depth, select, rng, false, 0u,
                           0u, [&](Light_sample const& ls) {
                               float const f = shading::phase_hg(shading::dot(wo, ls.dir), g);
                               float const w = ls.pdf / (ls.pdf * ls.pdf + f * f);
                               return (w * f) * (T * ls.radiance);
                           }, shadow, shadow2);
                float const x0 = rng.uniform();
                float const x1 = rng.uniform();
                float       pdf;
                V3 const    wi = shading::sample_hg(wo, g, x0, x1, pdf);
                p.ray_o[path]  = make_float4(pos.x, pos.y, pos.z, 0.f);
                p.ray_d[path]  = make_float4(wi.x, wi.y, wi.z, Ray_max_t);
                p.prev_n[path] = make_float4(0.f, 0.f, 1.f, 1.f);
                bsdf_pdf       = pdf;  // reflection / pdf == 1
                singular       = false;
                ++depth;
                ++vtx;
                extend = true;
            }
        } else if (!done) {
            uint32_t const inst = hit_instance(s, p, path);
            V3             vn[3];
            World_tri const wt = world_triangle(s, inst, id, vn);
            V3 const     a   = wt.a;
            V3 const     b   = wt.b;
            V3 const     c   = wt.c;
            float2 const uv  = p.hit_uv[path];
            float const  bw  = 1.f - uv.x - uv.y;
            V3 const     pos = bw * a + uv.x * b + uv.y * c;
            V3           geo_n = shading::normalize(shading::cross(b - a, c - a));
            V3           ns  = shading::normalize(bw * vn[0] + uv.x * vn[1] + uv.y * vn[2]);
            V3 const     wo  = -dir_in;
            uint32_t const mat_id = wt.material;
            shading::Material mat = s.materials[mat_id];
            if (mat.color_map | mat.surface_map) {
                float2 const t0  = s.uvs[wt.tri.x];
                float2 const t1  = s.uvs[wt.tri.y];
                float2 const t2  = s.uvs[wt.tri.z];
                float2 const tuv = make_float2(bw * t0.x + uv.x * t1.x + uv.y * t2.x,
                                               bw * t0.y + uv.x * t1.y + uv.y * t2.y);
                apply_texture_maps(s, mat, tuv, nearest_at_vertex(depth));
            }
            float const  cos_o = shading::dot(geo_n, wo);
            bool const   front = cos_o > 0.f;
            bool const   emits = mat.type == shading::Type_light;

            if (vtx > 0) {
                // Emission reached by the BSDF sample (connect_light, pathtracer_mis.cpp:349-380).
                if (emits) {
                    if (front || mat.two_sided) {
                        // only emitters registered as lights (su_create_light) are reached by
                        // a continuation ray; others are seen from the camera only
                        uint32_t const lb    = s.inst_shade[inst].light_base;
                        uint32_t const order = lb != 0xFFFFFFFFu ? s.light_order[lb + id] : 0xFFFFFFFFu;
                        float          w     = order != 0xFFFFFFFFu ? 1.f : 0.f;
                        if (!singular && order != 0xFFFFFFFFu) {
                            // the light-tree pick from the previous vertex (connect_light,
                            // pathtracer_mis.cpp:349-380)
                            float4 const pn    = p.prev_n[path];
                            float const  pick  = light_pick_pdf(s, f3v(ro), f3v(pn), pn.w != 0.f, order,
                                                                splits_at(s, depth));
                            float const  t     = p.hit_t[path];
                            float const  area  = s.light_tris[3 * order].w;
                            float const  pdf_l = pick * (t * t) / (fabsf(cos_o) * area);
                            w                  = power_heuristic(bsdf_pdf, pdf_l);
                        }
                        L = L + w * (T * mat.emission);
                    }
                    done = true;
                } else if (depth >= wave.max_bounces) {
                    done = true;
                } else if (depth >= wave.min_bounces) {
                    float const q = continuation_probability(wave, T);
                    if (rng.uniform() > q) {
                        done = true;
                    } else {
                        T = (1.f / q) * T;
                    }
                }
            } else if (emits) {
                // The camera sees the emitter directly.
                if (front || mat.two_sided) {
                    L = L + mat.emission;
                }
                done = true;
            }

            if (!done && mat.type == shading::Type_volume) {
                // Null boundary of a medium: the ray continues unchanged past the hit, the
                // medium changes (interface_change), depth and MIS state are kept
                // (pathtracer_mis.cpp:180-205, Straight_transmission).
                medium        = front ? mat_id + 1 : 0;
                p.ray_o[path] = make_float4(ro.x, ro.y, ro.z, offset_f(p.hit_t[path]));
                p.ray_d[path] = make_float4(rd.x, rd.y, rd.z, Ray_max_t);
                ++vtx;
                extend = true;
            } else if (!done && !front && !mat.two_sided) {
                done = true;  // back face of a one-sided material: no evaluation, no sample
            } else if (!done) {
                if (!front) {
                    geo_n = -geo_n;
                    ns    = -ns;
                }
                shading::Context ctx;
                ctx.frame = shading::make_frame(ns);
                ctx.geo_n = geo_n;
                ctx.wo    = wo;

                // The guide's mixture for this vertex (k_guide); continuation directions come
                // from it with probability gf, else from the BSDF, and every pdf the MIS
                // weights use is the combination of both.
                bool const  guided = wave.guiding && depth < wave.guide_depth && p.guide_ok[i];
                float const gf     = !guided ? 0.f : (mat.metallic == 1.f ? wave.metal_fraction : wave.guide_fraction);
                float4 const* const mix = reinterpret_cast<float4 const*>(p.guide_out + size_t(i) * Mixture_floats);

                // The first vertices sample from the pixel's golden ratio sequences (batch
                // rendering), the others from the path's random stream.
                bool const     golden  = wave.golden_n != 0 && depth < Golden_bounces;
                uint32_t const pixels  = launch->pixels;
                uint32_t const gview   = view_of(launch->view_offsets, launch->num_views, path % pixels);
                uint32_t const gpixel  = path % pixels - launch->view_offsets[gview];  // within its view
                uint32_t const gsample = wave.first_sample + path / pixels;

                // Next-event estimation (sample_lights / evaluate_light, pathtracer_mis.cpp:281-347).
                V3 const    ps     = offset_ray(pos, geo_n);
                float const select = golden ? golden_1d(wave, gpixel, gsample, golden_light_1d(depth, 0))
                                            : rng.uniform();
                next_event(s, p, wave, out, path, ps, geo_n, false, depth, select, rng, golden, gpixel, gsample,
                           [&](Light_sample const& ls) {
                               shading::Bxdf const f = shading::substitute_evaluate(mat, s.e_table, ctx, ls.dir);
                               float const pc = guided ? gf * mixture_pdf_at(mix, ls.dir) + (1.f - gf) * f.pdf
                                                       : f.pdf;
                               float const w  = ls.pdf / (ls.pdf * ls.pdf + pc * pc);
                               return w * (T * (ls.radiance * f.reflection));
                           }, shadow, shadow2);

                // Continuation direction: the BSDF sample (pathtracer_mis.cpp:153-201), or with
                // probability gf the guide's.  A guide direction gets the BSDF value and pdf the
                // BSDF sampler would give it -- below the geometric surface too, where the
                // Substitute BSDF (its cosines clamped to a small positive minimum) is not zero;
                // dropping those directions would bias the one-sample MIS estimate low.
                shading::Sampled smp;
                // With golden ratio sampling, the choice between guide and BSDF has a dimension
                // of its own, and the guide's lobe and direction use the BSDF's (one of the two
                // samplers is used at a vertex).
                float const choice = !guided ? 1.f
                                             : (golden ? golden_1d(wave, gpixel, gsample, golden_choice_1d(depth))
                                                       : rng.uniform());
                if (guided && choice < gf) {
                    float g0, g1, g2;
                    if (golden) {
                        g0              = golden_1d(wave, gpixel, gsample, golden_bsdf_1d(depth));
                        float2 const g2d = golden_2d(wave, gpixel, gsample, golden_bsdf_2d(depth));
                        g1              = g2d.x;
                        g2              = g2d.y;
                    } else {
                        g0 = rng.uniform();
                        g1 = rng.uniform();
                        g2 = rng.uniform();
                    }
                    smp.wi                = mixture_sample_at(mix, g0, g1, g2);
                    smp.specular          = false;
                    shading::Bxdf const f = shading::substitute_evaluate(mat, s.e_table, ctx, smp.wi);
                    smp.reflection        = f.reflection;
                    smp.pdf               = f.pdf;
                } else if (golden) {
                    float const  xl = golden_1d(wave, gpixel, gsample, golden_bsdf_1d(depth));
                    float2 const x2 = golden_2d(wave, gpixel, gsample, golden_bsdf_2d(depth));
                    smp = shading::substitute_sample(mat, s.e_table, ctx, xl, x2.x, x2.y);
                } else {
                    float const xl = rng.uniform();
                    float const x0 = rng.uniform();
                    float const x1 = rng.uniform();
                    smp = shading::substitute_sample(mat, s.e_table, ctx, xl, x0, x1);
                }
                if (smp.pdf > 0.f) {
                    float const pdf = guided && !smp.specular
                                          ? gf * mixture_pdf_at(mix, smp.wi) + (1.f - gf) * smp.pdf
                                          : smp.pdf;
                    if (guided && depth < wave.record_depth) {
                        // training record of this vertex (its radiance mark comes at the next)
                        uint32_t const r = path * wave.record_depth + depth;
                        float4* const  d = p.rec + size_t(r) * Record_float4;
                        d[0] = make_float4(pos.x, pos.y, pos.z, geo_n.x);
                        d[1] = make_float4(geo_n.y, geo_n.z, wo.x, wo.y);
                        d[2] = make_float4(wo.z, smp.wi.x, smp.wi.y, smp.wi.z);
                        d[3] = make_float4(T.x, T.y, T.z, 0.f);
                        d[4] = make_float4(0.f, 0.f, 0.f, 0.f);
                        p.open_record[path] = r;
                    }
                    V3 const o = offset_ray(pos, shading::dot(geo_n, smp.wi) > 0.f ? geo_n : -geo_n);
                    p.ray_o[path]  = make_float4(o.x, o.y, o.z, 0.f);
                    p.ray_d[path]  = make_float4(smp.wi.x, smp.wi.y, smp.wi.z, Ray_max_t);
                    p.prev_n[path] = make_float4(geo_n.x, geo_n.y, geo_n.z, 0.f);
                    T        = (1.f / pdf) * (T * smp.reflection);
                    bsdf_pdf = pdf;
                    singular = smp.specular;
                    ++depth;
                    ++vtx;
                    extend = true;
                }
            }
        }

        p.T[path]    = make_float4(T.x, T.y, T.z, bsdf_pdf);
        p.L[path]    = make_float4(L.x, L.y, L.z, 0.f);
        p.rng[path]  = rng.save();
        p.info[path] = pack_info(vtx, depth, singular, medium);
    }

    uint32_t const slot = append(out.count_out, extend);
    if (extend) {
        out.q_out[slot] = path;
    }
    uint32_t const sslot = append(out.count_shadow, shadow);
    if (shadow) {
        out.sq[sslot] = path;
    }
    uint32_t const sslot2 = append(out.count_shadow, shadow2);
    if (shadow2) {
        out.sq[sslot2] = path | Second_shadow;
    }
}

// ---- shadow rays through media: Worker::transmittance (rendering_worker.cpp:209-267) ----
// One shadow ray's walk from its origin: medium boundaries found by closest hits on boundary
// triangles, homogeneous segments adding their optical depth, density-grid segments
// multiplying in a ratio-tracking estimate (on a stream of its own, seeded from the path's
// state, which this kernel only reads: a vertex's shadow rays may be in flight together).
// Returns false when the ray is blocked; tr receives the transmittance.
template <bool Instances>
__device__ __forceinline__ bool walk_shadow(Scene_gpu const& s, Paths const& p, uint32_t path, float4 ro, float4 rd,
                                            uint32_t depth, uint32_t stream, uint32_t* overflow, V3& tr) {
    uint32_t medium = p.info[path] >> 17;
    float    t0     = ro.w;
    V3       tau    = v3(0.f, 0.f, 0.f);
    V3       w      = v3(1.f, 1.f, 1.f);
    bool     random = false;
    Rng      rng;
    uint2    stack[gpu::Stack_size];
    for (int crossing = 0; crossing < 64; ++crossing) {
        gpu::Ray_state      r;
        gpu::Traversal      tv;
        gpu::Instance_state is;
        gpu::start_ray(r, tv, make_float4(ro.x, ro.y, ro.z, t0), rd);
        if constexpr (Instances) {
            gpu::start_instances(r, is);
        }
        while (!gpu::traversal_step<false, true, Instances>(r, tv, stack, s.nodes, s.tris, s.hit_margin,
                                                            overflow, Class_surface, &is, s.inst_trace)) {
        }
        bool const  hit = r.best_id != gpu::Miss;
        float const end = hit ? r.tbest : rd.w;
        if (medium != 0) {
            shading::Material const m = s.materials[medium - 1];
            if (m.medium != 0) {
                if (!random) {
                    uint4 const st = p.rng[path];
                    rng.start((uint64_t(st.y) << 32) | st.x, (uint64_t(path) << 7) | stream);
                    random = true;
                }
                float const srs = shading::similarity_relation_scale(m.g, depth);
                if (!transmit_grid(s.media[m.medium - 1], m, srs, f3v(ro), f3v(rd), t0, end,
                                   nearest_at_vertex(depth), rng, w, s.tracking_capped)) {
                    return false;
                }
            } else {
                float const len = fmaxf(end - t0, 0.f);
                tau = tau + len * (m.mu_a + m.mu_s);
            }
        }
        if (!hit) {
            break;
        }
        World_tri const wt  = world_triangle(s, Instances ? is.best_inst : 0u, r.best_id);
        V3 const        geo = shading::cross(wt.b - wt.a, wt.c - wt.a);
        medium              = shading::dot(geo, v3(rd.x, rd.y, rd.z)) < 0.f ? wt.material + 1 : 0;
        t0                  = offset_f(r.tbest);
        if (t0 >= rd.w) {
            break;
        }
    }
    tr = v3(w.x * expf(-tau.x), w.y * expf(-tau.y), w.z * expf(-tau.z));
    return true;
}

// Shadow slots through media, one thread per entry: the queue holds `count` rays to emitters
// at its front and `env_count` rays to the environment at its back (entries capacity - 1
// downwards).  The light contribution times the transmittance is added to the path's radiance
// (L for the first slot, L2 for the second).  Picks take k_transmit_picks: a kernel of its own
// keeps this one free of branches on the entry's kind, which cost most of its lanes.
template <bool Instances = false>
__global__ void __launch_bounds__(Trace_block)
    k_transmit(Scene_gpu s, Paths p, uint32_t const* __restrict__ queue, uint32_t const* __restrict__ count,
               uint32_t const* __restrict__ env_count, uint32_t capacity, uint32_t* overflow) {
    uint32_t const j     = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t const front = *count;
    if (j >= front + *env_count) {
        return;
    }
    uint32_t const entry  = queue[j < front ? j : capacity - 1u - (j - front)];
    uint32_t const path   = entry & Entry_index;
    bool const     second = entry & Second_shadow;
    float4 const   ro     = second ? p.sh2_o[path] : p.sh_o[path];
    float4 const   rd     = second ? p.sh2_d[path] : p.sh_d[path];
    float4 const   c      = second ? p.sh2_L[path] : p.sh_L[path];
    V3             tr;
    if (!walk_shadow<Instances>(s, p, path, ro, rd, uint32_t(c.w), second ? 1u : 0u, overflow, tr)) {
        return;
    }
    float4* const Lp = second ? p.L2 : p.L;
    float4        l  = Lp[path];
    l.x += tr.x * c.x;
    l.y += tr.y * c.y;
    l.z += tr.z * c.z;
    Lp[path] = l;
}

// Picks through media, one thread per entry: the pick's contribution is scaled by the
// transmittance (zero when blocked) for k_pick_sum.
template <bool Instances = false>
__global__ void __launch_bounds__(Trace_block)
    k_transmit_picks(Scene_gpu s, Paths p, uint32_t const* __restrict__ queue, uint32_t const* __restrict__ count,
                     uint32_t* overflow) {
    uint32_t const j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= *count) {
        return;
    }
    uint32_t const pk  = queue[j] & Entry_index;
    float4 const   c   = p.pick_c[pk];
    uint32_t const rec = __float_as_uint(c.w);
    float4 const   o   = p.split_o[rec];
    uint4 const    m   = p.split_m[rec];
    V3             tr  = v3(0.f, 0.f, 0.f);
    if (!walk_shadow<Instances>(s, p, __float_as_uint(o.w), make_float4(o.x, o.y, o.z, 0.f), p.pick_d[pk], m.z,
                                2u + (pk - m.x), overflow, tr)) {
        tr = v3(0.f, 0.f, 0.f);
    }
    p.pick_c[pk] = make_float4(tr.x * c.x, tr.y * c.y, tr.z * c.z, c.w);
}

// ---- film: Filtered_1p0::add_sample (sensor/filtered.inl:125-187) as a gather ----
__constant__ float c_filter[Filter_samples];

__device__ __forceinline__ float filter_weight(float d) {
    float const x  = fminf(d * d, 1.f) * float(Filter_samples - 1);
    int const   o  = int(x);
    float const t  = x - float(o);
    int const   o1 = o + 1 < Filter_samples ? o + 1 : Filter_samples - 1;
    return c_filter[o] + t * (c_filter[o1] - c_filter[o]);
}

__global__ void k_gather(Paths p, Launch const* __restrict__ launch, uint32_t film_pixels, uint32_t samples,
                         float4* film, float4* comp) {
    uint32_t const q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= film_pixels) {
        return;
    }
    uint32_t const view   = view_of(launch->film_offsets, launch->num_views, q);
    uint32_t const w      = launch->cams[view].w;
    uint32_t const local  = q - launch->film_offsets[view];
    int const      x      = int(local % w);
    int const      y      = int(local / w);
    uint32_t const bw     = w + 2 * Film_border;
    uint32_t const base   = launch->view_offsets[view];  // the view's first bordered pixel
    uint32_t const traced = launch->pixels;               // bordered pixels per sample slot
    float4         acc    = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int dy = -1; dy <= 1; ++dy) {
        uint32_t const sy = uint32_t(y - dy + Film_border);  // bordered row, always inside
        for (int dx = -1; dx <= 1; ++dx) {
            uint32_t const src = base + sy * bw + uint32_t(x - dx + Film_border);
            for (uint32_t k = 0; k < samples; ++k) {
                uint32_t const path = k * traced + src;
                float2 const   uv   = p.puv[path];
                float const    wt   = filter_weight(uv.x - 0.5f - float(dx)) *
                                 filter_weight(uv.y - 0.5f - float(dy));
                float4 const L  = p.L[path];
                float4 const L2 = p.L2[path];
                acc.x += wt * (L.x + L2.x);
                acc.y += wt * (L.y + L2.y);
                acc.z += wt * (L.z + L2.z);
                acc.w += wt;
            }
        }
    }
    // Kahan-compensated accumulation into the frame's film.
    float4 sum = film[q];
    float4 c   = comp[q];
    float4 yv  = make_float4(acc.x - c.x, acc.y - c.y, acc.z - c.z, acc.w - c.w);
    float4 t   = make_float4(sum.x + yv.x, sum.y + yv.y, sum.z + yv.z, sum.w + yv.w);
    comp[q]    = make_float4((t.x - sum.x) - yv.x, (t.y - sum.y) - yv.y, (t.z - sum.z) - yv.z,
                          (t.w - sum.w) - yv.w);
    film[q]    = t;
}

// ---- guide training: samples from the wave's records ----
// Batch entry i takes record hash(i, pass) of the wave; a finished record (radiance mark set)
// gives the input encoding, the continuation direction and the weight
// luminance((L_final - L_mark) / T): the continuation's radiance times f cos / pdf at the
// vertex, the target of the product-guiding loss.  Other records, and rows past the batch up to
// the tile boundary, give weight 0 and zero inputs.  The inputs are written as the training
// kernel reads them (BF16 tiles of 128 rows); each block adds its weights in a fixed order into
// parts[block] (the loss is normalised by their total).
__global__ void __launch_bounds__(256)
    k_train_gather(Paths p, Launch const* __restrict__ launch, uint32_t records, uint32_t batch,
                   uint32_t const* __restrict__ pass_counter, __nv_bfloat16* in, float* dir, float* weight,
                   float* parts) {
    Wave const&      wave = launch->wave;
    uint32_t const   pass = *pass_counter;
    __shared__ float part[256];
    uint32_t const   i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t const   rows = (batch + guide::Tile - 1) / guide::Tile * guide::Tile;
    float            w    = 0.f;
    float            enc[guide::Inputs];
    if (i < batch) {
        uint64_t const h = (uint64_t(i) * 0x9E3779B97F4A7C15ull) ^ (uint64_t(pass + 1) * 0xD1B54A32D192ED03ull);
        uint32_t const r = uint32_t(((h ^ (h >> 29)) * 0xBF58476D1CE4E5B9ull >> 32) % records);
        float4 const*  d = p.rec + size_t(r) * Record_float4;
        float4 const   mark = d[4];
        float4 const   a = d[0], b = d[1], c = d[2], t = d[3];
        if (mark.w == 1.f) {
            uint32_t const path = r / wave.record_depth;
            float4 const   l    = p.L[path];
            float4 const   l2   = p.L2[path];
            float const    cx   = t.x > 0.f ? (l.x + l2.x - mark.x) / t.x : 0.f;
            float const    cy   = t.y > 0.f ? (l.y + l2.y - mark.y) / t.y : 0.f;
            float const    cz   = t.z > 0.f ? (l.z + l2.z - mark.z) / t.z : 0.f;
            // AP1 (ACEScg) luminance
            float const lum = 0.2722287f * cx + 0.6740818f * cy + 0.0536895f * cz;
            w               = (lum > 0.f && lum < 1e30f) ? lum : 0.f;
        }
        guide::encode(box_coordinates(wave, v3(a.x, a.y, a.z)), v3(a.w, b.x, b.y), v3(b.z, b.w, c.x), enc);
        dir[3 * size_t(i)]     = w > 0.f ? c.y : 0.f;
        dir[3 * size_t(i) + 1] = w > 0.f ? c.z : 0.f;
        dir[3 * size_t(i) + 2] = w > 0.f ? c.w : 1.f;
        weight[i]              = w;
    }
    if (i < rows) {
        __nv_bfloat16* const tile = in + size_t(i / guide::Tile) * guide::Tile * guide::Inputs;
        int const            r    = int(i % guide::Tile);
#pragma unroll
        for (int k = 0; k < guide::Inputs; k += 8) {
            __nv_bfloat162 h[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                h[j] = __floats2bfloat162_rn(w > 0.f ? enc[k + 2 * j] : 0.f, w > 0.f ? enc[k + 2 * j + 1] : 0.f);
            }
            *reinterpret_cast<uint4*>(tile + guide::tiled(r, k, guide::Inputs)) = *reinterpret_cast<uint4*>(h);
        }
    }
    part[threadIdx.x] = w;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (int(threadIdx.x) < o) {
            part[threadIdx.x] += part[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        parts[blockIdx.x] = part[0];
    }
}

// ---- hero-wavelength spectral transport (spectral.cuh): one persistent launch ----
// The renderer's spectral mode, for scenes of participating media, emitters and the
// environment (the many-view volume workload): each thread takes (view, pixel, sample) work
// items from a counter and traces the whole path carrying Hero_count wavelengths; every RGB
// quantity (emission, medium coefficients) is upsampled at them.  Tracking is the RGB
// renderer's spectral-MIS delta tracking over the carried wavelengths (majorants from the RGB
// coefficients, which bound every upsampled value since the basis is a partition of unity);
// light selection picks one light (no splitting); shadow rays walk their medium crossings
// with ratio tracking and are blocked by any other triangle.  Each sample's radiance is read
// out to ACEScg (c_spec_resp) and splatted with the film filter into its view's film with
// atomics (so the film's summation order, unlike the wavefront renderer's, is not fixed).
namespace spec = spb::spectral;
constexpr int Spec_table = 341;  // readout at 1 nm steps over [Lambda_min, Lambda_max]
__constant__ float c_spec_resp[3 * Spec_table];

// The sample's film colour: sum over the carried wavelengths of radiance times the readout
// (which includes the round-trip correction and Lambda_span / Hero_count).
__device__ __forceinline__ V3 spec_readout(spec::V4 L, spec::V4 lambdas) {
    V3 acc = v3(0.f, 0.f, 0.f);
    for (int k = 0; k < spec::Hero_count; ++k) {
        float const x = lambdas.v[k] - spec::Lambda_min;
        int const   i = min(max(int(x), 0), Spec_table - 2);
        float const f = x - float(i);
        acc.x += L.v[k] * ((1.f - f) * c_spec_resp[3 * i] + f * c_spec_resp[3 * i + 3]);
        acc.y += L.v[k] * ((1.f - f) * c_spec_resp[3 * i + 1] + f * c_spec_resp[3 * i + 4]);
        acc.z += L.v[k] * ((1.f - f) * c_spec_resp[3 * i + 2] + f * c_spec_resp[3 * i + 5]);
    }
    return acc;
}

__device__ __forceinline__ spec::V4 spec_of(V3 c, spec::V4 lambdas) {
    return spec::upsample(c.x, c.y, c.z, lambdas);
}

__device__ __forceinline__ bool spec_below_abort(spec::V4 w) {
    return spec::maximum(w) < Abort_epsilon;
}

// Delta tracking with spectral MIS in a homogeneous medium (track_homogeneous over the
// carried wavelengths).
__device__ bool spec_track_homogeneous(spec::V4 mu_a, spec::V4 mu_s, float t, float d, Rng& rng, float& t_out,
                                       spec::V4& lw, uint32_t* capped) {
    spec::V4 const mu_t = spec::add(mu_a, mu_s);
    float const    mt   = spec::maximum(mu_t);
    lw                  = spec::splat(1.f);
    if (!(mt > 1e-10f)) {
        return false;
    }
    float const imt  = 1.f / mt;
    spec::V4    mu_n = spec::add(spec::splat(mt), spec::scale(-1.f, mu_t));
    for (int step = 0; step < Max_tracking_steps; ++step) {
        t -= logf(1.f - rng.uniform()) * imt;
        if (t > d) {
            return false;
        }
        float const ms = spec::average(spec::mul(mu_s, lw));
        float const mn = spec::average(spec::mul(mu_n, lw));
        float const mc = ms + mn;
        if (mc < 1e-10f) {
            return false;
        }
        float const ps = ms / mc;
        float const pn = mn / mc;
        if ((rng.uniform() <= 1.f - pn) & (ps > 0.f)) {
            lw    = spec::mul(lw, spec::scale(1.f / (mt * ps), mu_s));
            t_out = t;
            return true;
        }
        lw = spec::mul(lw, spec::scale(1.f / (mt * pn), mu_n));
    }
    atomicAdd(capped, 1u);
    return false;
}

// Delta tracking with spectral MIS through a density grid (track_grid over the carried
// wavelengths); maj_t bounds the coefficients at density 1 for every wavelength.
__device__ bool spec_track_grid(Medium_gpu const& g, float maj_t, spec::V4 mu_a, spec::V4 mu_s, V3 ro, V3 rd,
                                float t0, float t1, Rng& rng, float& t_out, spec::V4& lw, uint32_t* capped) {
    V3 const o     = to_texture(g, ro);
    V3 const d     = to_texture_dir(g, rd);
    lw             = spec::splat(1.f);
    int  steps     = 0;
    bool scattered = false;
    walk_cells(g, o, d, t0, t1, [&](float2 cell, float ta, float tb) {
        float const mt = cell.y * maj_t;
        if (mt < Min_mt) {
            return false;
        }
        float const imt = 1.f / mt;
        for (float t = ta; steps < Max_tracking_steps; ++steps) {
            t -= logf(1.f - rng.uniform()) * imt;
            if (t > tb) {
                return false;
            }
            float const    den  = sample_density(g, o + t * d);
            spec::V4 const ms3  = spec::scale(den, mu_s);
            spec::V4 const mu_n = spec::add(spec::splat(mt), spec::scale(-den, spec::add(mu_a, mu_s)));
            float const    ms   = spec::average(spec::mul(ms3, lw));
            float const    mn   = spec::average(spec::mul(mu_n, lw));
            float const    sum  = ms + mn;
            if (!(sum > 0.f)) {
                lw = spec::splat(0.f);
                return true;
            }
            float const ps = ms / sum;
            float const pn = mn / sum;
            if ((rng.uniform() <= 1.f - pn) & (ps > 0.f)) {
                lw        = spec::mul(lw, spec::scale(1.f / (mt * ps), ms3));
                t_out     = t;
                scattered = true;
                return true;
            }
            lw = spec::mul(lw, spec::scale(1.f / (mt * pn), mu_n));
        }
        return true;
    });
    if (steps >= Max_tracking_steps) {
        atomicAdd(capped, 1u);
    }
    return scattered;
}

// Ratio tracking through a density grid (transmit_grid over the carried wavelengths): w is
// multiplied by the estimate; false when it falls below Abort_epsilon.
__device__ bool spec_transmit_grid(Medium_gpu const& g, float maj_t, float min_t, spec::V4 mu_t, V3 ro, V3 rd,
                                   float t0, float t1, Rng& rng, spec::V4& w, uint32_t* capped) {
    V3 const o       = to_texture(g, ro);
    V3 const d       = to_texture_dir(g, rd);
    int      steps   = 0;
    bool     blocked = false;
    walk_cells(g, o, d, t0, t1, [&](float2 cell, float ta, float tb) {
        float const mt = cell.y * maj_t;
        if (mt < Min_mt) {
            return false;
        }
        float const cm = fmaxf(cell.x * min_t, 0.f);
        if (cm > 0.f) {
            w = spec::scale(expf(-(tb - ta) * cm), w);
            if (spec_below_abort(w)) {
                blocked = true;
                return true;
            }
        }
        float const mr = mt - cm;
        if (mr < Min_mt) {
            return false;
        }
        float const imr = 1.f / mr;
        for (float t = ta; steps < Max_tracking_steps; ++steps) {
            t -= logf(1.f - rng.uniform()) * imr;
            if (t > tb) {
                return false;
            }
            float const den = sample_density(g, o + t * d);
            for (int k = 0; k < spec::Hero_count; ++k) {
                w.v[k] *= (mr - (den * mu_t.v[k] - cm)) * imr;
            }
            if (spec_below_abort(w)) {
                blocked = true;
                return true;
            }
        }
        return false;
    });
    if (steps >= Max_tracking_steps) {
        atomicAdd(capped, 1u);
    }
    return !blocked;
}

// The medium coefficients of material index + 1 `medium` at the carried wavelengths, with the
// similarity-relation scale of scattering at depth (shading::similarity_relation_scale).
struct Spec_medium {
    spec::V4 mu_a, mu_s;
    float    maj_t, min_t;  // bounds of mu_t at density 1 over every wavelength
};

__device__ __forceinline__ Spec_medium spec_medium(shading::Material const& m, uint32_t depth, spec::V4 lambdas) {
    float const srs = shading::similarity_relation_scale(m.g, depth);
    V3 const    ms  = srs * m.mu_s;
    Spec_medium r;
    r.mu_a  = spec_of(m.mu_a, lambdas);
    r.mu_s  = spec_of(ms, lambdas);
    r.maj_t = shading::max_component(m.mu_a) + shading::max_component(ms);
    r.min_t = shading::min_component(m.mu_a) + shading::min_component(ms);
    return r;
}

// Transmittance of a shadow ray from o along d up to dist, starting inside `medium`: medium
// boundaries are crossed, any other triangle blocks it.
__device__ bool spec_transmit(Scene_gpu const& s, V3 o, V3 d, float dist, uint32_t medium, uint32_t depth,
                              spec::V4 lambdas, Rng& rng, uint2* stack, uint32_t* overflow, spec::V4& tr) {
    tr       = spec::splat(1.f);
    float t0 = 0.f;
    for (int crossing = 0; crossing < 64; ++crossing) {
        gpu::Ray_state r;
        gpu::Traversal tv;
        gpu::start_ray(r, tv, make_float4(o.x, o.y, o.z, t0), make_float4(d.x, d.y, d.z, dist));
        while (!gpu::traversal_step<false>(r, tv, stack, s.nodes, s.tris, s.hit_margin, overflow)) {
        }
        bool const  hit = r.best_id != gpu::Miss;
        float const end = hit ? r.tbest : dist;
        if (medium != 0) {
            shading::Material const m  = s.materials[medium - 1];
            Spec_medium const       sm = spec_medium(m, depth, lambdas);
            if (m.medium != 0) {
                if (!spec_transmit_grid(s.media[m.medium - 1], sm.maj_t, sm.min_t, spec::add(sm.mu_a, sm.mu_s), o, d,
                                        t0, end, rng, tr, s.tracking_capped)) {
                    return false;
                }
            } else {
                float const len = fmaxf(end - t0, 0.f);
                for (int k = 0; k < spec::Hero_count; ++k) {
                    tr.v[k] *= expf(-len * (sm.mu_a.v[k] + sm.mu_s.v[k]));
                }
            }
        }
        if (!hit) {
            return true;
        }
        World_tri const wt = world_triangle(s, 0u, r.best_id);
        if (s.materials[wt.material].type != shading::Type_volume) {
            return false;
        }
        V3 const geo = shading::cross(wt.b - wt.a, wt.c - wt.a);
        medium       = shading::dot(geo, d) < 0.f ? wt.material + 1 : 0;
        t0           = offset_f(r.tbest);
        if (t0 >= dist) {
            return true;
        }
    }
    return true;
}

// Adds a sample's colour to the film pixels its filter footprint covers (the splat form of
// k_gather's gather: a sample of bordered pixel (sx, sy) at offset uv adds weight
// f(u - 0.5 - dx) f(v - 0.5 - dy) to film pixel (sx + dx, sy + dy)).
__device__ __forceinline__ void spec_splat(float4* film, uint32_t film_base, int w, int h, int sx, int sy, float u,
                                           float v, V3 c) {
    for (int dy = -1; dy <= 1; ++dy) {
        int const fy = sy + dy;
        if (fy < 0 || fy >= h) {
            continue;
        }
        float const wy = filter_weight(v - 0.5f - float(dy));
        for (int dx = -1; dx <= 1; ++dx) {
            int const fx = sx + dx;
            if (fx < 0 || fx >= w) {
                continue;
            }
            float const  wt  = wy * filter_weight(u - 0.5f - float(dx));
            float* const dst = reinterpret_cast<float*>(film + film_base + uint32_t(fy) * uint32_t(w) + uint32_t(fx));
            atomicAdd(dst + 0, wt * c.x);
            atomicAdd(dst + 1, wt * c.y);
            atomicAdd(dst + 2, wt * c.z);
            atomicAdd(dst + 3, wt);
        }
    }
}

// ---- phase guiding at medium vertices (spectral mode; no counterpart in the reference) ----
// A grid of cells over the scene box, each with one vMF lobe of the directions radiance
// arrives from at the medium vertices inside it.  A training pass records, per scattering
// vertex, the radiance the path later receives through the direction it left by (divided by
// the throughput up to that direction), and sums weight x direction and weight per cell; a fit
// turns the sums into a lobe (mean direction; concentration from the mean resultant length,
// Banerjee et al. 2005).  Guided passes draw the continuation from the lobe with probability
// `fraction` and from the Henyey-Greenstein phase function otherwise (one-sample MIS: the
// weight is phase / mixture pdf, and the mixture pdf weighs light hits and next-event
// estimation), so the estimate stays unbiased whatever the lobes are.
struct Phase_guide {
    float4*       sums;    // per cell while training: (sum w d, sum w)
    uint32_t*     counts;  // per cell while training: directions recorded
    float4 const* lobes;   // per cell after the fit: (mean direction, kappa); kappa 0: no lobe
    float4        lo;      // scene box origin
    float4        scale;   // cells per world unit on each axis
    int           n;       // cells per axis
    float         fraction;
};

constexpr int   Phase_cells      = 32;   // per axis
constexpr int   Phase_ring       = 3;    // vertices a training path credits
constexpr int   Phase_min_count  = 16;   // directions a cell needs for a lobe
constexpr float Phase_kappa_max  = 64.f;

__device__ __forceinline__ uint32_t phase_cell(Phase_guide const& g, V3 p) {
    int const x = min(max(int((p.x - g.lo.x) * g.scale.x), 0), g.n - 1);
    int const y = min(max(int((p.y - g.lo.y) * g.scale.y), 0), g.n - 1);
    int const z = min(max(int((p.z - g.lo.z) * g.scale.z), 0), g.n - 1);
    return uint32_t((z * g.n + y) * g.n + x);
}

// One cell's lobe from its sums.
__global__ void k_phase_fit(Phase_guide g, float4* lobes) {
    uint32_t const c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= uint32_t(g.n * g.n * g.n)) {
        return;
    }
    float4 const sm = g.sums[c];
    float4       l  = make_float4(0.f, 0.f, 1.f, 0.f);
    float const  m  = sqrtf(sm.x * sm.x + sm.y * sm.y + sm.z * sm.z);
    if (g.counts[c] >= uint32_t(Phase_min_count) && sm.w > 0.f && m > 0.f) {
        float const r = fminf(m / sm.w, 0.999f);
        l = make_float4(sm.x / m, sm.y / m, sm.z / m, fminf(r * (3.f - r * r) / (1.f - r * r), Phase_kappa_max));
    }
    lobes[c] = l;
}

// Kinds of spectral launch: plain, training the phase guide, guided by it.
constexpr int Spectral_plain = 0, Spectral_train = 1, Spectral_guided = 2;

template <int Mode>
__global__ void __launch_bounds__(Trace_block)
    k_spectral(Scene_gpu s, Launch const* __restrict__ launch, uint64_t total, unsigned long long* next, float4* film,
               uint32_t* overflow, unsigned long long* counts, Phase_guide guide) {
    Wave const     wave   = launch->wave;
    uint32_t const pixels = launch->pixels;
    uint2          stack[gpu::Stack_size];
    unsigned long long segments = 0, shadows = 0;
    for (;;) {
        unsigned long long const item = atomicAdd(next, 1ull);
        if (item >= total) {
            break;
        }
        uint32_t const pixel       = uint32_t(item % pixels);
        uint32_t const slot        = uint32_t(item / pixels);
        uint32_t const view        = view_of(launch->view_offsets, launch->num_views, pixel);
        Cam const      cam         = launch->cams[view];
        uint32_t const local       = pixel - launch->view_offsets[view];
        uint32_t const view_pixels = launch->view_offsets[view + 1] - launch->view_offsets[view];
        uint32_t const bw          = cam.w + 2 * Film_border;
        int const      px          = int(local % bw) - Film_border;
        int const      py          = int(local / bw) - Film_border;
        Rng            rng;
        rng.start(wave.seed, uint64_t(local) + uint64_t(wave.first_sample + slot) * view_pixels);
        float const u  = rng.uniform();
        float const v  = rng.uniform();
        float const cx = float(px) + u;
        float const cy = float(py) + v;
        V3          d  = v3(cam.left_top.x + cx * cam.d_x.x + cy * cam.d_y.x, cam.left_top.y + cx * cam.d_x.y + cy * cam.d_y.y,
                            cam.left_top.z + cx * cam.d_x.z + cy * cam.d_y.z);
        d              = shading::normalize(d);
        d = v3(d.x * cam.r0.x + d.y * cam.r1.x + d.z * cam.r2.x, d.x * cam.r0.y + d.y * cam.r1.y + d.z * cam.r2.y,
               d.x * cam.r0.z + d.y * cam.r1.z + d.z * cam.r2.z);
        spec::V4 const lambdas = spec::wavelengths(rng.uniform());
        spec::V4       T       = spec::splat(1.f);
        spec::V4       L       = spec::splat(0.f);
        V3             o       = v3(cam.pos.x, cam.pos.y, cam.pos.z);
        float          tmin    = 0.f;
        uint32_t       medium  = 0;
        uint32_t       depth   = 0;
        bool           camera  = true;  // no scattering vertex yet
        float          pdf_prev = 0.f;  // phase pdf of the last continuation
        V3             prev_p   = o;    // its vertex
        // training: the last Phase_ring vertices (newest first), their cell, direction, inverse
        // throughput and the radiance credited to them
        uint32_t ring_cell[Phase_ring];
        V3       ring_dir[Phase_ring];
        float    ring_inv[Phase_ring];
        float    ring_acc[Phase_ring];
        for (int k = 0; k < Phase_ring; ++k) {
            ring_cell[k] = 0xFFFFFFFFu;
            ring_dir[k]  = v3(0.f, 0.f, 0.f);
            ring_inv[k]  = 0.f;
            ring_acc[k]  = 0.f;
        }
        auto const credit = [&](spec::V4 dl) {  // radiance the path received after the ring's vertices
            if constexpr (Mode == Spectral_train) {
                float const x = spec::average(dl);
                for (int k = 0; k < Phase_ring; ++k) {
                    ring_acc[k] += x * ring_inv[k];
                }
            }
        };
        auto const deposit = [&](int k) {
            if constexpr (Mode == Spectral_train) {
                if (ring_cell[k] != 0xFFFFFFFFu && ring_acc[k] > 0.f && isfinite(ring_acc[k])) {
                    float* const sm = reinterpret_cast<float*>(guide.sums + ring_cell[k]);
                    atomicAdd(sm + 0, ring_acc[k] * ring_dir[k].x);
                    atomicAdd(sm + 1, ring_acc[k] * ring_dir[k].y);
                    atomicAdd(sm + 2, ring_acc[k] * ring_dir[k].z);
                    atomicAdd(sm + 3, ring_acc[k]);
                }
                if (ring_cell[k] != 0xFFFFFFFFu) {
                    atomicAdd(guide.counts + ring_cell[k], 1u);
                }
            }
        };
        for (int seg = 0; seg < 1024; ++seg) {
            ++segments;
            gpu::Ray_state r;
            gpu::Traversal tv;
            gpu::start_ray(r, tv, make_float4(o.x, o.y, o.z, tmin), make_float4(d.x, d.y, d.z, Ray_max_t));
            while (!gpu::traversal_step<false>(r, tv, stack, s.nodes, s.tris, s.hit_margin, overflow)) {
            }
            bool const  hit   = r.best_id != gpu::Miss;
            float const t_hit = hit ? r.tbest : Ray_max_t;
            bool        scattered = false;
            float       t_sc      = 0.f;
            if (medium != 0) {
                shading::Material const m  = s.materials[medium - 1];
                Spec_medium const       sm = spec_medium(m, depth, lambdas);
                spec::V4                lw;
                scattered = m.medium != 0 ? spec_track_grid(s.media[m.medium - 1], sm.maj_t, sm.mu_a, sm.mu_s, o, d,
                                                             tmin, t_hit, rng, t_sc, lw, s.tracking_capped)
                                          : spec_track_homogeneous(sm.mu_a, sm.mu_s, tmin, t_hit, rng, t_sc, lw,
                                                                   s.tracking_capped);
                T = spec::mul(T, lw);
                if (spec_below_abort(lw)) {
                    break;
                }
            }
            if (scattered) {
                // A scattering vertex in the medium (HG phase function).
                if (depth >= wave.max_bounces) {
                    break;
                }
                if (depth >= wave.min_bounces) {
                    // unbiased Russian roulette: a throughput above 1 (spectral MIS and guide
                    // weights can reach it) always continues
                    float const q = fminf(spec::maximum(T), 1.f);
                    if (rng.uniform() > q) {
                        break;
                    }
                    T = spec::scale(1.f / q, T);
                }
                shading::Material const m   = s.materials[medium - 1];
                float const             g   = shading::van_de_hulst_anisotropy(m.g, depth);
                V3 const                pos = o + t_sc * d;
                V3 const                wo  = -d;
                // the cell's lobe and its share of the continuation (guided launches)
                guide::Lobe lobe{v3(0.f, 0.f, 1.f), 0.f, 0.f};
                if constexpr (Mode == Spectral_guided) {
                    float4 const l = guide.lobes[phase_cell(guide, pos)];
                    if (l.w > 0.f) {
                        lobe = guide::Lobe{v3(l.x, l.y, l.z), l.w, guide.fraction};
                    }
                }
                auto const mixture = [&](V3 wi, float f) {  // pdf of the continuation proposal
                    return lobe.weight > 0.f ? (1.f - lobe.weight) * f + lobe.weight * guide::vmf_pdf(lobe, wi) : f;
                };
                float const             select = rng.uniform();
                float const             r1     = rng.uniform();
                float const             r2     = rng.uniform();
                Light_pick              pick[1];
                if (select_lights(s, pos, v3(0.f, 0.f, 1.f), true, select, false, pick) == 1) {
                    Light_sample ls;
                    if (sample_light(s, pos, v3(0.f, 0.f, 1.f), true, pick[0], r1, r2, rng, ls)) {
                        float const f  = shading::phase_hg(shading::dot(wo, ls.dir), g);
                        float const pc = mixture(ls.dir, f);
                        float const w  = ls.pdf / (ls.pdf * ls.pdf + pc * pc);
                        spec::V4    tr;
                        ++shadows;
                        if (spec_transmit(s, pos, ls.dir, ls.dist, medium, depth, lambdas, rng, stack, overflow, tr)) {
                            spec::V4 const dl =
                                spec::mul(spec::scale(w * f, T), spec::mul(tr, spec_of(ls.radiance, lambdas)));
                            L = spec::add(L, dl);
                            credit(dl);
                        }
                    }
                }
                float       pdf;
                bool const  from_lobe = lobe.weight > 0.f && rng.uniform() < lobe.weight;
                float const x0        = rng.uniform();
                float const x1        = rng.uniform();
                V3          wi;
                if (from_lobe) {
                    wi = guide::vmf_sample(lobe, x0, x1);
                    pdf = shading::phase_hg(shading::dot(wo, wi), g);
                } else {
                    wi = shading::sample_hg(wo, g, x0, x1, pdf);
                }
                float const pm = mixture(wi, pdf);  // pdf is the phase value here
                if (!(pm > 0.f)) {
                    break;
                }
                T = spec::scale(pdf / pm, T);
                if constexpr (Mode == Spectral_train) {
                    deposit(Phase_ring - 1);
                    for (int k = Phase_ring - 1; k > 0; --k) {
                        ring_cell[k] = ring_cell[k - 1];
                        ring_dir[k]  = ring_dir[k - 1];
                        ring_inv[k]  = ring_inv[k - 1];
                        ring_acc[k]  = ring_acc[k - 1];
                    }
                    // the incident radiance along wi, importance-weighted by 1 / pdf of the phase
                    // sample, so that the lobe follows the radiance rather than the phase function
                    float const tavg = spec::average(T);
                    ring_cell[0] = phase_cell(guide, pos);
                    ring_dir[0]  = wi;
                    ring_inv[0]  = tavg > 0.f && pdf > 0.f ? 1.f / (tavg * pdf) : 0.f;
                    ring_acc[0]  = 0.f;
                }
                o        = pos;
                d        = wi;
                tmin     = 0.f;
                pdf_prev = pm;
                prev_p   = pos;
                camera   = false;
                ++depth;
                continue;
            }
            if (!hit) {
                // The environment: seen by the camera; by continuations when it is a light,
                // weighted against its next-event pdf (the sphere of directions at a medium vertex).
                if (medium == 0 && (camera || s.env.w > 0.f)) {
                    float w = 1.f;
                    if (!camera) {
                        w = power_heuristic(pdf_prev, s.env.w * (1.f / (4.f * shading::Pi)));
                    }
                    spec::V4 const dl = spec::scale(w, spec::mul(T, spec_of(v3(s.env.x, s.env.y, s.env.z), lambdas)));
                    L                 = spec::add(L, dl);
                    credit(dl);
                }
                break;
            }
            World_tri const         wt    = world_triangle(s, 0u, r.best_id);
            shading::Material const mat   = s.materials[wt.material];
            V3 const                geo   = shading::normalize(shading::cross(wt.b - wt.a, wt.c - wt.a));
            float const             cos_o = -shading::dot(geo, d);
            bool const              front = cos_o > 0.f;
            if (mat.type == shading::Type_light) {
                if (front || mat.two_sided) {
                    uint32_t const lb    = s.inst_shade[0].light_base;
                    uint32_t const order = lb != 0xFFFFFFFFu ? s.light_order[lb + r.best_id] : 0xFFFFFFFFu;
                    float          w     = camera ? 1.f : (order != 0xFFFFFFFFu ? 1.f : 0.f);
                    if (!camera && order != 0xFFFFFFFFu) {
                        float const pick  = light_pick_pdf(s, prev_p, v3(0.f, 0.f, 1.f), true, order, false);
                        float const area  = s.light_tris[3 * order].w;
                        float const t     = r.tbest;  // the ray starts at the vertex prev_p
                        float const pdf_l = pick * (t * t) / (fabsf(cos_o) * area);
                        w                 = power_heuristic(pdf_prev, pdf_l);
                    }
                    spec::V4 const dl = spec::scale(w, spec::mul(T, spec_of(mat.emission, lambdas)));
                    L                 = spec::add(L, dl);
                    credit(dl);
                }
                break;
            }
            // A medium boundary (the only other material of a spectral scene): the ray
            // continues past it in the medium behind it.
            medium = front ? wt.material + 1 : 0;
            tmin   = offset_f(r.tbest);
        }
        spec_splat(film, launch->film_offsets[view], int(cam.w), int(cam.h), px, py, u, v, spec_readout(L, lambdas));
        for (int k = 0; k < Phase_ring; ++k) {
            deposit(k);
        }
    }
    atomicAdd(counts, segments);
    atomicAdd(counts + 1, shadows);
}

__global__ void k_resolve(float4 const* film, float4 const* comp, uint32_t n, float4* out) {
    uint32_t const q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) {
        return;
    }
    float4 const s  = film[q];
    float4 const c  = comp[q];
    double const wt = double(s.w) - double(c.w);
    double const iw = wt > 0.0 ? 1.0 / wt : 0.0;
    out[q] = make_float4(float((double(s.x) - double(c.x)) * iw), float((double(s.y) - double(c.y)) * iw),
                         float((double(s.z) - double(c.z)) * iw), 1.f);
}

}  // namespace

struct Renderer::Device {
    // scene
    uint4*             nodes      = nullptr;
    float4*            tris       = nullptr;
    uint4*             tri_info   = nullptr;
    float4*            positions  = nullptr;
    float4*            normals    = nullptr;
    shading::Material* materials  = nullptr;
    float4*            light_nodes = nullptr;
    float4*            light_cones = nullptr;
    float4*            light_tris  = nullptr;
    uint32_t*          light_order = nullptr;
    float*             e_table    = nullptr;
    Medium_gpu*        media      = nullptr;
    gpu::Instance_trace* inst_trace     = nullptr;
    Instance_shade*      inst_shade     = nullptr;
    uint32_t*            inst_materials = nullptr;
    bool                 instanced      = false;  // two-level trees
    uint32_t             per_sm_flat    = 1;      // traversal blocks per SM (occupancy), flat trees
    uint32_t             per_sm_inst    = 1;      // ... two-level trees
    float2*              uvs            = nullptr;
    Texture_gpu*         textures       = nullptr;
    std::vector<float4*> texture_texels;
    uint32_t*            golden_sorted  = nullptr;  // frac(j / phi) * 2^32, j < golden_n, ascending
    uint32_t             golden_n       = 0;
    std::vector<float*>  grid_density;  // one per density grid
    std::vector<float2*> grid_cells;
    Volume_light_gpu*    volume_lights  = nullptr;  // emitting media that are lights
    Emission_dist_gpu*   emission_dists = nullptr;
    std::vector<float*>  dist_data;  // per emission distribution: prob, cdf_z, cdf_y, cdf_x
    float4*              blackbody      = nullptr;  // 16 per medium: emission by temperature
    float4*              phase_sums     = nullptr;  // spectral mode's phase guide (Phase_guide)
    uint32_t*            phase_counts   = nullptr;
    float4*              phase_lobes    = nullptr;
    // the light tree's nodes as uploaded, and the splitting threshold their split radii are for
    std::vector<float>   light_tree_nodes;
    float                split_radii_threshold = -1.f;
    uint32_t           num_lights = 0;
    float4             env        = {0.f, 0.f, 0.f, 0.f};
    float              hit_margin = 0.f;
    float4             bounds_lo  = {0.f, 0.f, 0.f, 0.f};  // scene box (guide encoding)
    float4             bounds_inv = {1.f, 1.f, 1.f, 0.f};
    // path guiding
    guide::Network     net;
    bool               net_ready     = false;
    uint32_t           guide_grid    = 1;      // k_guide blocks (persistent)
    Tuner              tuner;
    uint32_t           sms           = 1;
    // per-wave launch block (pinned host copy, device copy) and the captured wave graphs
    Launch*            launch_host   = nullptr;
    Launch*            launch_dev    = nullptr;
    struct Wave_graph {
        uint32_t        k, trace_grid, iterations, events;
        cudaGraphExec_t exec;  // nullptr: seen once, not captured yet
    };
    std::vector<Wave_graph> graphs;
    cudaEvent_t        wave_ev[2]    = {nullptr, nullptr};
    // event pairs around the guide's inference and training launches of one render call
    std::vector<cudaEvent_t> guide_events;
    uint32_t           guide_paths   = 0;  // paths the guide buffers hold
    uint32_t           guide_records = 0;  // record depth they were sized for
    uint32_t           train_capacity = 0;
    __nv_bfloat16*     train_in    = nullptr;  // the batch's inputs, BF16 tiles of 128
    float*             train_dir   = nullptr;
    float*             train_w     = nullptr;
    float*             train_parts = nullptr;  // per gather block: its weights' sum
    uint32_t*          pass_counter = nullptr;  // training batches drawn since the network was set
    // one captured training pass (guide_steps x [gather, gradients, Adam]) and its shape
    struct Train_graph {
        uint32_t        records, batch, steps;
        float           lr;
        cudaGraphExec_t exec;
    };
    Train_graph        train_graph{0, 0, 0, 0.f, nullptr};
    // paths
    uint32_t  capacity = 0;
    Paths     paths{};
    uint32_t* queue[2] = {nullptr, nullptr};
    uint32_t* shadow_queue   = nullptr;
    uint32_t* transmit_queue      = nullptr;  // shadow slots through media (2 per path)
    uint32_t* transmit_pick_queue = nullptr;  // picks through media
    uint32_t* counters       = nullptr;
    uint32_t* pinned_count   = nullptr;  // host-pinned word for the queue-length check
    bool      has_media      = false;
    // split light selection: the most lights one selection returns in this scene, the depth
    // the split walk starts at, and the picks the buffers hold
    uint32_t  max_picks        = 1;
    // spectral mode: the scene holds only emitters and non-emissive media; the readout table is
    // uploaded; the work counter and the kernel's step counts
    bool                spectral_scene = false;
    bool                spectral_table = false;
    unsigned long long* spectral_work  = nullptr;
    uint32_t  split_depth_bias = 0;
    uint64_t  pick_capacity    = 0;
    // film
    float4*   film = nullptr;
    float4*   comp = nullptr;
    float4*   out  = nullptr;
    uint32_t  film_pixels = 0;    // film pixels of all views
    // the views: cameras, prefix tables of their bordered (sampled) and film pixels
    Cam*      cams          = nullptr;
    uint32_t* view_offsets  = nullptr;
    uint32_t* film_offsets  = nullptr;
    uint32_t  num_views     = 0;
    uint32_t  traced_pixels = 0;
    int       trace_grid  = 0;
    cudaStream_t stream   = nullptr;
    cudaEvent_t  ev0      = nullptr;
    cudaEvent_t  ev1      = nullptr;
};

namespace {

// The renderer's device buffers come from the device's default stream-ordered memory pool,
// set to keep the memory it gets back (release threshold: unlimited): an engine created after
// another was released, or a wave larger than the last, reuses that memory instead of having
// the driver map (and, on release, unmap) gigabytes anew -- which took up to half a second per
// frame.  Allocation and release are ordered on the legacy default stream and completed before
// they return, so the buffers behave as cudaMalloc'd ones for every stream.
cudaError_t pool_malloc(void** p, size_t bytes) {
    static bool const keep = [] {
        int           dev  = 0;
        cudaMemPool_t pool = nullptr;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t threshold = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
        }
        return true;
    }();
    (void)keep;
    cudaError_t const e = cudaMallocAsync(p, bytes, 0);
    return e == cudaSuccess ? cudaStreamSynchronize(0) : e;
}

template <typename T>
cudaError_t dev_malloc(T** p, size_t bytes) {
    return pool_malloc(reinterpret_cast<void**>(p), bytes);
}

// Returns a buffer to the pool once the device is idle (no kernel may still use it).
template <typename T>
void free_ptr(T*& p) {
    if (p) {
        cudaDeviceSynchronize();
        cudaFreeAsync(p, 0);
        cudaStreamSynchronize(0);
        p = nullptr;
    }
}

template <typename T>
cudaError_t upload(T*& dst, void const* src, size_t bytes) {
    free_ptr(dst);
    cudaError_t e = dev_malloc(&dst, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) {
        return e;
    }
    return bytes ? cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
}

// Majorant cells of a density grid, one thread per cell: (min, max) density over its
// Cell_dim^3 block of voxels plus one voxel on every side (wrapped for the repeat address mode,
// clipped otherwise), the minimum starting at 1 as in Octree_builder::Splitter::split
// (volumetric_octree_builder.cpp:170-186).
__global__ void k_majorant_cells(float const* __restrict__ density, int nx, int ny, int nz, int cx, int cy, int cz,
                                 bool repeat, float2* cells) {
    int const i = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= cx * cy * cz) {
        return;
    }
    int const n[3] = {nx, ny, nz};
    int const c[3] = {i % cx, (i / cx) % cy, i / (cx * cy)};
    int const dim  = 1 << Cell_log2;
    int       lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = c[a] * dim - 1;
        hi[a] = min((c[a] + 1) * dim + 1, n[a] + (repeat ? 1 : 0));
        if (!repeat) {
            lo[a] = max(lo[a], 0);
        }
    }
    auto const wrap = [&](int v, int axis) { return ((v % n[axis]) + n[axis]) % n[axis]; };
    float      mn   = 1.f;
    float      mx   = 0.f;
    for (int z = lo[2]; z < hi[2]; ++z) {
        for (int y = lo[1]; y < hi[1]; ++y) {
            size_t const row = (size_t(wrap(z, 2)) * n[1] + wrap(y, 1)) * n[0];
            for (int x = lo[0]; x < hi[0]; ++x) {
                float const v = __ldg(density + row + wrap(x, 0));
                mn            = fminf(mn, v);
                mx            = fmaxf(mx, v);
            }
        }
    }
    if (mn > mx) {
        mn = mx = 0.f;
    }
    cells[i] = make_float2(mn, mx);
}

// The emission distribution of a density grid whose voxels emit density x emission, or
// density x the emission at the voxel's temperature, times the second channel of a
// two-channel density (Grid_emission::prepare_sampling,
// volumetric_grid.cpp:182-318, built with
// SU_IBL_MIS_COMPENSATION): voxel weights max(luminance - 0.6 average luminance, 0) (ACEScg
// luminance) normalised to probabilities, with the cumulative sums over slices, rows and voxels
// the device draws from (Distribution_3D over Distribution_2D over Distribution_1D).
struct Emission_dist_host {
    std::vector<float> data;  // prob (n), cdf_z (nz + 1), cdf_y (nz (ny + 1)), cdf_x (nz ny (nx + 1))
    uint32_t           dims[3] = {0, 0, 0};
    bool               repeat  = false;  // the grid's address mode
    double             average[3] = {0.0, 0.0, 0.0};  // mean emitted radiance over the voxels
    double             total      = 0.0;              // sum of the weights (0: nothing to draw)
};

Emission_dist_host emission_distribution(Density_grid const& g, V3 emission, float const* temperature,
                                         float4 const* blackbody, float const* scale) {
    size_t const nx = g.dims[0], ny = g.dims[1], nz = g.dims[2], n = nx * ny * nz;
    auto const   lum = [](double r, double gg, double b) {
        return 0.2722287168 * r + 0.6740817658 * gg + 0.0536895174 * b;
    };
    Emission_dist_host  out;
    std::copy(g.dims, g.dims + 3, out.dims);
    std::vector<double> w(n);
    double              sum[3] = {0.0, 0.0, 0.0};
    for (size_t v = 0; v < n; ++v) {
        double const d = double(g.density[v]) * (scale ? scale[v] : 1.f);
        V3 const     e = temperature ? blackbody_emission(blackbody, temperature[v]) : emission;
        sum[0] += d * e.x;
        sum[1] += d * e.y;
        sum[2] += d * e.z;
        w[v] = lum(d * e.x, d * e.y, d * e.z);
    }
    for (int k = 0; k < 3; ++k) {
        out.average[k] = sum[k] / double(n);
    }
    double const al = 0.6 * lum(out.average[0], out.average[1], out.average[2]);
    for (double& x : w) {
        x = std::max(x - al, 0.0);
        out.total += x;
    }
    if (!(out.total > 0.0)) {
        return out;
    }
    out.data.resize(n + (nz + 1) + nz * (ny + 1) + nz * ny * (nx + 1));
    float* const prob  = out.data.data();
    float* const cdf_z = prob + n;
    float* const cdf_y = cdf_z + (nz + 1);
    float* const cdf_x = cdf_y + nz * (ny + 1);
    // A running sum normalised by its total, ending at exactly 1 (uniform where the total is 0;
    // such a range is never drawn).
    auto const cumulate = [](double const* x, size_t len, double total, float* cdf) {
        double acc = 0.0;
        cdf[0]     = 0.f;
        for (size_t i = 0; i < len; ++i) {
            acc += x[i];
            cdf[i + 1] = total > 0.0 ? float(acc / total) : float(double(i + 1) / double(len));
        }
        cdf[len] = 1.f;
    };
    std::vector<double> slice(nz, 0.0), row(nz * ny, 0.0);
    for (size_t z = 0; z < nz; ++z) {
        for (size_t y = 0; y < ny; ++y) {
            double const* r = &w[(z * ny + y) * nx];
            double        s = 0.0;
            for (size_t x = 0; x < nx; ++x) {
                s += r[x];
                prob[(z * ny + y) * nx + x] = float(r[x] / out.total);
            }
            row[z * ny + y] = s;
            slice[z] += s;
            cumulate(r, nx, s, cdf_x + (z * ny + y) * (nx + 1));
        }
        cumulate(&row[z * ny], ny, slice[z], cdf_y + z * (ny + 1));
    }
    cumulate(slice.data(), nz, out.total, cdf_z);
    return out;
}

}  // namespace

void Renderer::free_grids() {
    for (float*& g : d_->grid_density) {
        free_ptr(g);
    }
    for (float2*& c : d_->grid_cells) {
        free_ptr(c);
    }
    d_->grid_density.clear();
    d_->grid_cells.clear();
    free_ptr(d_->media);
    for (float*& e : d_->dist_data) {
        free_ptr(e);
    }
    d_->dist_data.clear();
    free_ptr(d_->volume_lights);
    free_ptr(d_->emission_dists);
    free_ptr(d_->blackbody);
}

Renderer::Renderer() : d_(new Device) {
    float table[Filter_samples];
    float const alpha = 1.8f;
    float const tail  = std::exp(-alpha);
    for (int i = 0; i < Filter_samples; ++i) {
        float const x = float(i) / float(Filter_samples - 1);
        table[i]      = std::max(0.f, std::exp(-alpha * x) - tail);
    }
    cudaMemcpyToSymbol(c_filter, table, sizeof(table));
    cudaStreamCreateWithFlags(&d_->stream, cudaStreamNonBlocking);
    cudaMallocHost(&d_->pinned_count, sizeof(uint32_t));
    cudaEventCreate(&d_->ev0);
    cudaEventCreate(&d_->ev1);
    int per_sm = 0;
    int sms    = 0;
    int dev    = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace<false>, Trace_block, 0);
    int per_sm_inst = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_inst, k_trace<false, false, true>, Trace_block, 0);
    d_->per_sm_flat = uint32_t(std::max(1, per_sm));
    d_->per_sm_inst = uint32_t(std::max(1, per_sm_inst));
    d_->trace_grid = std::max(1, per_sm) * std::max(1, sms);
    d_->sms        = uint32_t(std::max(1, sms));
    d_->tuner.reset(uint32_t(std::max(1, per_sm)));
    cudaEventCreate(&d_->wave_ev[0]);
    cudaEventCreate(&d_->wave_ev[1]);
}

Renderer::~Renderer() {
    if (!d_) {
        return;
    }
    cudaDeviceSynchronize();
    free_ptr(d_->train_in);
    free_ptr(d_->train_dir);
    free_ptr(d_->train_w);
    free_ptr(d_->train_parts);
    free_ptr(d_->pass_counter);
    free_ptr(d_->nodes);
    free_ptr(d_->tris);
    free_ptr(d_->tri_info);
    free_ptr(d_->positions);
    free_ptr(d_->normals);
    free_ptr(d_->materials);
    free_ptr(d_->light_nodes);
    free_ptr(d_->light_cones);
    free_ptr(d_->light_tris);
    free_ptr(d_->light_order);
    free_ptr(d_->e_table);
    free_ptr(d_->inst_trace);
    free_ptr(d_->inst_shade);
    free_ptr(d_->inst_materials);
    free_ptr(d_->golden_sorted);
    free_ptr(d_->uvs);
    free_ptr(d_->textures);
    for (float4*& t : d_->texture_texels) {
        free_ptr(t);
    }
    free_grids();
    Paths& p = d_->paths;
    free_ptr(p.ray_o);
    free_ptr(p.ray_d);
    free_ptr(p.hit_id);
    free_ptr(p.hit_inst);
    free_ptr(p.hit_t);
    free_ptr(p.hit_uv);
    free_ptr(p.T);
    free_ptr(p.L);
    free_ptr(p.puv);
    free_ptr(p.rng);
    free_ptr(p.info);
    free_ptr(p.sh_o);
    free_ptr(p.sh_d);
    free_ptr(p.sh_L);
    free_ptr(p.prev_n);
    free_ptr(p.split_o);
    free_ptr(p.sh2_o);
    free_ptr(p.sh2_d);
    free_ptr(p.sh2_L);
    free_ptr(p.split_m);
    free_ptr(p.pick_d);
    free_ptr(p.pick_c);
    free_ptr(p.L2);
    free_ptr(p.guide_in);
    free_ptr(p.guide_out);
    free_ptr(p.guide_ok);
    free_ptr(p.rec);
    free_ptr(p.open_record);
    d_->guide_paths = 0;
    free_ptr(d_->queue[0]);
    free_ptr(d_->queue[1]);
    free_ptr(d_->shadow_queue);
    free_ptr(d_->transmit_queue);
    free_ptr(d_->transmit_pick_queue);
    free_ptr(d_->counters);
    if (d_->pinned_count) {
        cudaFreeHost(d_->pinned_count);
    }
    free_ptr(d_->film);
    free_ptr(d_->comp);
    free_ptr(d_->out);
    free_ptr(d_->cams);
    free_ptr(d_->spectral_work);
    free_ptr(d_->phase_sums);
    free_ptr(d_->phase_counts);
    free_ptr(d_->phase_lobes);
    free_ptr(d_->view_offsets);
    free_ptr(d_->film_offsets);
    if (d_->stream) {
        cudaStreamDestroy(d_->stream);
    }
    cudaEventDestroy(d_->ev0);
    cudaEventDestroy(d_->ev1);
    for (cudaEvent_t e : d_->guide_events) {
        cudaEventDestroy(e);
    }
    cudaEventDestroy(d_->wave_ev[0]);
    cudaEventDestroy(d_->wave_ev[1]);
    for (auto const& g : d_->graphs) {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
        }
    }
    free_ptr(d_->launch_dev);
    if (d_->launch_host) {
        cudaFreeHost(d_->launch_host);
    }
    delete d_;
}

int32_t Renderer::fail_cuda(char const* what, int code) {
    error_ = std::string(what) + ": " + cudaGetErrorString(cudaError_t(code));
    return SPB_ERROR_CUDA;
}

#define SPB_RCUDA(call)                                   \
    do {                                                  \
        cudaError_t const e_ = (call);                    \
        if (e_ != cudaSuccess) {                          \
            return fail_cuda(#call, int(e_));             \
        }                                                 \
    } while (0)

int32_t Renderer::set_scene(Scene_desc const& scene, uint32_t num_threads) {
    clear_graphs();
    if (scene.instances.empty()) {
        error_ = "scene has no triangles";
        return SPB_ERROR_STATE;
    }
    for (Instance_desc const& in : scene.instances) {
        if (in.mesh >= scene.meshes.size() || scene.meshes[in.mesh].indices.empty()) {
            error_ = "instance of a missing or empty mesh";
            return SPB_ERROR_ARGUMENT;
        }
    }
    auto const material_of = [&](Instance_desc const& in, uint32_t slot) {
        uint32_t const m = slot < in.materials.size() ? in.materials[slot] : in.fallback;
        return m < scene.materials.size() ? m : in.fallback;
    };
    // Two levels when flattening would multiply the distinct meshes' triangles (unless the
    // scene's "instancing" setting decides).
    uint64_t              flat_tris = 0;
    uint64_t              mesh_tris = 0;
    std::vector<uint32_t> uses(scene.meshes.size(), 0);
    for (Instance_desc const& in : scene.instances) {
        flat_tris += scene.meshes[in.mesh].indices.size() / 3;
        if (uses[in.mesh]++ == 0) {
            mesh_tris += scene.meshes[in.mesh].indices.size() / 3;
        }
    }
    bool const two_level = scene.instancing == 1 ||
                           (scene.instancing < 0 && flat_tris > 4 * mesh_tris && flat_tris > (1u << 20));
    if (flat_tris >= (1ull << 32)) {
        error_ = "scene has too many triangles";
        return SPB_ERROR_ARGUMENT;
    }
    d_->instanced = two_level;
    // A new scene is tuned anew, at the occupancy of the traversal it uses.
    d_->tuner.reset(two_level ? d_->per_sm_inst : d_->per_sm_flat);
    d_->has_media      = false;
    d_->spectral_scene = !two_level;

    std::vector<Wide_node>           nodes;
    std::vector<Wide_triangle>       tris;
    std::vector<uint4>               info;    // per triangle: vertices, material slot
    std::vector<float4>              pos;     // object space (world space when flattened)
    std::vector<float4>              nrm;
    std::vector<float2>              uv;      // texture coordinates, parallel to pos
    std::vector<uint32_t>            inst_materials;
    std::vector<Instance_shade>      shade;
    std::vector<gpu::Instance_trace> trace;
    std::vector<Light_input>         emitters;
    uint32_t                         light_slots = 0;
    double                           lo[3] = {1e300, 1e300, 1e300};
    double                           hi[3] = {-1e300, -1e300, -1e300};
    uint64_t                         device_triangles = 0;

    // An emissive triangle of a light prop, with its world-space vertices.
    auto const add_emitter = [&](double const a[3], double const b[3], double const c[3],
                                 shading::Material const& m, uint32_t slot, uint32_t material) {
        Light_input li;
        for (int k = 0; k < 3; ++k) {
            li.a[k] = a[k];
            li.b[k] = b[k];
            li.c[k] = c[k];
        }
        double const e1[3] = {li.b[0] - li.a[0], li.b[1] - li.a[1], li.b[2] - li.a[2]};
        double const e2[3] = {li.c[0] - li.a[0], li.c[1] - li.a[1], li.c[2] - li.a[2]};
        double const cx    = e1[1] * e2[2] - e1[2] * e2[1];
        double const cy    = e1[2] * e2[0] - e1[0] * e2[2];
        double const cz    = e1[0] * e2[1] - e1[1] * e2[0];
        double const area  = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
        li.two_sided       = m.two_sided != 0;
        // Light::power (light.cpp:38-48) and Scene::light_power (scene.cpp:504): area times the
        // largest radiance component, twice that for two-sided emitters.
        li.power = area * std::max({double(m.emission.x), double(m.emission.y), double(m.emission.z)}) *
                   (li.two_sided ? 2.0 : 1.0);
        li.slot     = slot;
        li.material = material;
        if (area > 0.0 && li.power > 0.0) {
            emitters.push_back(li);
        }
    };
    auto const grow = [&](double const p[3]) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], p[k]);
            hi[k] = std::max(hi[k], p[k]);
        }
    };

    if (!two_level) {
        // Every instance flattened into world space (one tree); shading sees one identity
        // instance whose material slots are the materials themselves.
        std::vector<float>    wpos;
        std::vector<uint32_t> windex;
        std::vector<uint32_t> tri_class;
        for (Instance_desc const& in : scene.instances) {
            Mesh_desc const& mesh = scene.meshes[in.mesh];
            uint32_t const   base = uint32_t(wpos.size() / 3);
            float const*     m    = in.trafo;
            float const*     rot  = in.rotation;
            for (size_t v = 0; v < mesh.positions.size() / 3; ++v) {
                float const x = mesh.positions[3 * v];
                float const y = mesh.positions[3 * v + 1];
                float const z = mesh.positions[3 * v + 2];
                // row vector times matrix: p' = x * row0 + y * row1 + z * row2 + row3
                float const wx = x * m[0] + y * m[4] + z * m[8] + m[12];
                float const wy = x * m[1] + y * m[5] + z * m[9] + m[13];
                float const wz = x * m[2] + y * m[6] + z * m[10] + m[14];
                wpos.push_back(wx);
                wpos.push_back(wy);
                wpos.push_back(wz);
                pos.push_back(make_float4(wx, wy, wz, 0.f));
                uv.push_back(mesh.uvs.size() >= 2 * (v + 1) ? make_float2(mesh.uvs[2 * v], mesh.uvs[2 * v + 1])
                                                            : make_float2(0.f, 0.f));
                float const nx = mesh.normals[3 * v];
                float const ny = mesh.normals[3 * v + 1];
                float const nz = mesh.normals[3 * v + 2];
                nrm.push_back(make_float4(nx * rot[0] + ny * rot[3] + nz * rot[6], nx * rot[1] + ny * rot[4] + nz * rot[7],
                                          nx * rot[2] + ny * rot[5] + nz * rot[8], 0.f));
                double const wp[3] = {wx, wy, wz};
                grow(wp);
            }
            for (size_t t = 0; t < mesh.indices.size() / 3; ++t) {
                uint32_t const mat = material_of(in, mesh.tri_slot[t]);
                uint32_t const v[3] = {base + mesh.indices[3 * t], base + mesh.indices[3 * t + 1],
                                       base + mesh.indices[3 * t + 2]};
                uint32_t const global = uint32_t(info.size());
                info.push_back(make_uint4(v[0], v[1], v[2], mat));
                windex.insert(windex.end(), v, v + 3);
                shading::Material const& sm = scene.materials[mat];
                bool const volume = sm.type == shading::Type_volume;
                d_->has_media |= volume;
                d_->spectral_scene &= sm.type == shading::Type_light ||
                                      (volume && !(sm.emission.x > 0.f || sm.emission.y > 0.f || sm.emission.z > 0.f) &&
                                       !(sm.medium != 0 && scene.media[sm.medium - 1].color[0] != 0));
                tri_class.push_back(volume ? Class_boundary : Class_surface);
                if (in.light && sm.type == shading::Type_light) {
                    double a[3], b[3], c[3];
                    for (int k = 0; k < 3; ++k) {
                        a[k] = wpos[3 * size_t(v[0]) + k];
                        b[k] = wpos[3 * size_t(v[1]) + k];
                        c[k] = wpos[3 * size_t(v[2]) + k];
                    }
                    add_emitter(a, b, c, sm, global, mat);
                }
            }
        }
        Wide_bvh    bvh;
        std::string err;
        if (!build_wide_bvh(uint32_t(pos.size()), uint32_t(info.size()), wpos.data(), windex.data(), num_threads,
                            bvh, err, tri_class.data())) {
            error_ = "BVH build: " + err;
            return SPB_ERROR_ARGUMENT;
        }
        nodes          = std::move(bvh.nodes);
        tris           = std::move(bvh.triangles);
        d_->hit_margin = bvh.hit_margin;
        Instance_shade id{};
        id.o2w[0] = make_float4(1.f, 0.f, 0.f, 0.f);
        id.o2w[1] = make_float4(0.f, 1.f, 0.f, 0.f);
        id.o2w[2] = make_float4(0.f, 0.f, 1.f, 0.f);
        id.nrm[0] = id.o2w[0];
        id.nrm[1] = id.o2w[1];
        id.nrm[2] = id.o2w[2];
        shade.push_back(id);
        inst_materials.resize(scene.materials.size());
        for (uint32_t k = 0; k < inst_materials.size(); ++k) {
            inst_materials[k] = k;
        }
        light_slots      = uint32_t(info.size());
        device_triangles = info.size();
    } else {
        // One tree per (mesh, per-triangle class) in object space, a top-level tree over the
        // instances' world boxes.
        struct Blas {
            std::vector<Wide_node>     nodes;
            std::vector<Wide_triangle> tris;
            float                      margin;
            uint32_t                   depth;
            uint32_t                   node_off = 0;
            uint32_t                   tri_off  = 0;
        };
        std::vector<Blas>                                      blases;
        std::map<std::pair<uint32_t, std::vector<uint32_t>>, uint32_t> blas_of;
        std::vector<uint32_t>                                  inst_blas(scene.instances.size());
        std::vector<uint32_t>                                  mesh_vbase(scene.meshes.size(), 0xFFFFFFFFu);
        std::vector<uint32_t>                                  mesh_tbase(scene.meshes.size(), 0);
        std::vector<float>                                     boxes(6 * scene.instances.size());
        for (size_t i = 0; i < scene.instances.size(); ++i) {
            Instance_desc const& in   = scene.instances[i];
            Mesh_desc const&     mesh = scene.meshes[in.mesh];
            uint32_t const       nt   = uint32_t(mesh.indices.size() / 3);
            if (mesh_vbase[in.mesh] == 0xFFFFFFFFu) {
                mesh_vbase[in.mesh] = uint32_t(pos.size());
                mesh_tbase[in.mesh] = uint32_t(info.size());
                for (size_t v = 0; v < mesh.positions.size() / 3; ++v) {
                    pos.push_back(make_float4(mesh.positions[3 * v], mesh.positions[3 * v + 1], mesh.positions[3 * v + 2], 0.f));
                    nrm.push_back(make_float4(mesh.normals[3 * v], mesh.normals[3 * v + 1], mesh.normals[3 * v + 2], 0.f));
                    uv.push_back(mesh.uvs.size() >= 2 * (v + 1) ? make_float2(mesh.uvs[2 * v], mesh.uvs[2 * v + 1])
                                                                : make_float2(0.f, 0.f));
                }
                uint32_t const vb = mesh_vbase[in.mesh];
                for (uint32_t t = 0; t < nt; ++t) {
                    info.push_back(make_uint4(vb + mesh.indices[3 * t], vb + mesh.indices[3 * t + 1],
                                              vb + mesh.indices[3 * t + 2], mesh.tri_slot[t]));
                }
            }
            std::vector<uint32_t> cls(nt);
            uint32_t              max_slot = 0;
            for (uint32_t t = 0; t < nt; ++t) {
                bool const volume = scene.materials[material_of(in, mesh.tri_slot[t])].type == shading::Type_volume;
                d_->has_media |= volume;
                cls[t]   = volume ? Class_boundary : Class_surface;
                max_slot = std::max(max_slot, mesh.tri_slot[t]);
            }
            auto key = std::make_pair(in.mesh, cls);
            auto it  = blas_of.find(key);
            if (it == blas_of.end()) {
                Wide_bvh    bvh;
                std::string err;
                if (!build_wide_bvh(uint32_t(mesh.positions.size() / 3), nt, mesh.positions.data(),
                                    mesh.indices.data(), num_threads, bvh, err, cls.data())) {
                    error_ = "BVH build: " + err;
                    return SPB_ERROR_ARGUMENT;
                }
                Blas b;
                b.nodes  = std::move(bvh.nodes);
                b.tris   = std::move(bvh.triangles);
                b.margin = bvh.hit_margin;
                b.depth  = bvh.max_depth;
                it       = blas_of.emplace(std::move(key), uint32_t(blases.size())).first;
                blases.push_back(std::move(b));
            }
            inst_blas[i] = it->second;

            // Maps: object -> world (row vectors times trafo), its inverse, the normals' rotation.
            float const* m = in.trafo;
            double       L[3][3], tr[3];
            for (int r = 0; r < 3; ++r) {
                for (int c = 0; c < 3; ++c) {
                    L[r][c] = m[4 * r + c];
                }
                tr[r] = m[12 + r];
            }
            double const det = L[0][0] * (L[1][1] * L[2][2] - L[1][2] * L[2][1]) -
                               L[0][1] * (L[1][0] * L[2][2] - L[1][2] * L[2][0]) +
                               L[0][2] * (L[1][0] * L[2][1] - L[1][1] * L[2][0]);
            if (!(std::fabs(det) > 1e-30)) {
                error_ = "instance with a singular transformation";
                return SPB_ERROR_ARGUMENT;
            }
            double Li[3][3];  // inverse of L
            Li[0][0] = (L[1][1] * L[2][2] - L[1][2] * L[2][1]) / det;
            Li[0][1] = (L[0][2] * L[2][1] - L[0][1] * L[2][2]) / det;
            Li[0][2] = (L[0][1] * L[1][2] - L[0][2] * L[1][1]) / det;
            Li[1][0] = (L[1][2] * L[2][0] - L[1][0] * L[2][2]) / det;
            Li[1][1] = (L[0][0] * L[2][2] - L[0][2] * L[2][0]) / det;
            Li[1][2] = (L[0][2] * L[1][0] - L[0][0] * L[1][2]) / det;
            Li[2][0] = (L[1][0] * L[2][1] - L[1][1] * L[2][0]) / det;
            Li[2][1] = (L[0][1] * L[2][0] - L[0][0] * L[2][1]) / det;
            Li[2][2] = (L[0][0] * L[1][1] - L[0][1] * L[1][0]) / det;
            // world_j = sum_i object_i L[i][j] + tr_j; object_k = sum_j Li[j][k] (world_j - tr_j)
            gpu::Instance_trace it_rec{};
            Instance_shade      sh{};
            for (int k = 0; k < 3; ++k) {
                double const off = -(Li[0][k] * tr[0] + Li[1][k] * tr[1] + Li[2][k] * tr[2]);
                it_rec.w2o[k]    = make_float4(float(Li[0][k]), float(Li[1][k]), float(Li[2][k]), float(off));
                sh.o2w[k]        = make_float4(m[k], m[4 + k], m[8 + k], m[12 + k]);
                sh.nrm[k]        = make_float4(in.rotation[k], in.rotation[3 + k], in.rotation[6 + k], 0.f);
            }
            it_rec.hit_margin = blases[inst_blas[i]].margin;
            trace.push_back(it_rec);
            sh.tri_base = mesh_tbase[in.mesh];
            sh.mat_base = uint32_t(inst_materials.size());
            for (uint32_t k = 0; k <= max_slot; ++k) {
                inst_materials.push_back(material_of(in, k));
            }
            sh.light_base = 0xFFFFFFFFu;
            bool const emits = in.light && std::any_of(mesh.tri_slot.begin(), mesh.tri_slot.end(), [&](uint32_t k) {
                                   return scene.materials[material_of(in, k)].type == shading::Type_light;
                               });
            if (emits) {
                sh.light_base = light_slots;
                light_slots += nt;
            }
            shade.push_back(sh);

            // World box of the instance (its transformed vertices) and its emitters.
            std::vector<double> wv(mesh.positions.size());
            double blo[3] = {1e300, 1e300, 1e300}, bhi[3] = {-1e300, -1e300, -1e300};
            for (size_t v = 0; v < mesh.positions.size() / 3; ++v) {
                double const x = mesh.positions[3 * v], y = mesh.positions[3 * v + 1], z = mesh.positions[3 * v + 2];
                for (int k = 0; k < 3; ++k) {
                    wv[3 * v + k] = x * L[0][k] + y * L[1][k] + z * L[2][k] + tr[k];
                    blo[k]        = std::min(blo[k], wv[3 * v + k]);
                    bhi[k]        = std::max(bhi[k], wv[3 * v + k]);
                }
                grow(&wv[3 * v]);
            }
            for (int k = 0; k < 3; ++k) {
                boxes[6 * i + k]     = std::nextafter(float(blo[k]), -INFINITY);
                boxes[6 * i + 3 + k] = std::nextafter(float(bhi[k]), INFINITY);
            }
            if (emits) {
                for (uint32_t t = 0; t < nt; ++t) {
                    uint32_t const           mat = material_of(in, mesh.tri_slot[t]);
                    shading::Material const& sm  = scene.materials[mat];
                    if (sm.type == shading::Type_light) {
                        add_emitter(&wv[3 * size_t(mesh.indices[3 * t])], &wv[3 * size_t(mesh.indices[3 * t + 1])],
                                    &wv[3 * size_t(mesh.indices[3 * t + 2])], sm, sh.light_base + t, mat);
                    }
                }
            }
        }
        Wide_bvh    top;
        std::string err;
        if (!build_wide_instances(uint32_t(scene.instances.size()), boxes.data(), Class_instance, num_threads, top,
                                  err)) {
            error_ = "top-level tree: " + err;
            return SPB_ERROR_ARGUMENT;
        }
        uint32_t deepest = 0;
        nodes            = std::move(top.nodes);
        tris             = std::move(top.triangles);
        for (Blas& b : blases) {
            b.node_off = uint32_t(nodes.size());
            b.tri_off  = uint32_t(tris.size());
            for (Wide_node n : b.nodes) {
                n.child_base += b.node_off;
                n.tri_base += b.tri_off;
                nodes.push_back(n);
            }
            tris.insert(tris.end(), b.tris.begin(), b.tris.end());
            deepest = std::max(deepest, b.depth);
            device_triangles += b.tris.size();
        }
        if (top.max_depth + deepest + 2 > Max_wide_depth) {
            error_ = "top-level and instance trees together deeper than the traversal stack";
            return SPB_ERROR_ARGUMENT;
        }
        for (size_t i = 0; i < scene.instances.size(); ++i) {
            trace[i].root = blases[inst_blas[i]].node_off;
        }
        d_->hit_margin = top.hit_margin;
    }
    stats_.instances        = two_level ? uint32_t(scene.instances.size()) : 0u;
    stats_.device_triangles = device_triangles;
    instances_        = stats_.instances;
    device_triangles_ = device_triangles;

    cudaDeviceSynchronize();
    SPB_RCUDA(upload(d_->nodes, nodes.data(), nodes.size() * sizeof(Wide_node)));
    SPB_RCUDA(upload(d_->tris, tris.data(), tris.size() * sizeof(Wide_triangle)));
    SPB_RCUDA(upload(d_->inst_shade, shade.data(), shade.size() * sizeof(Instance_shade)));
    SPB_RCUDA(upload(d_->inst_materials, inst_materials.data(), inst_materials.size() * sizeof(uint32_t)));
    free_ptr(d_->inst_trace);
    if (!trace.empty()) {
        SPB_RCUDA(upload(d_->inst_trace, trace.data(), trace.size() * sizeof(gpu::Instance_trace)));
    }

    // Emitting media of light props (Scene::create_light, scene.cpp:330-350).  The medium of a
    // built-in Cube is a light that next-event estimation samples inside (Light::Type::Volume for
    // a homogeneous medium, Volume_image for a density grid); another shape's medium cannot be
    // sampled there (Shape::sample_volume fails and pdf_volume is 0 for it), so its emission
    // counts with weight 1 on every segment, as does that of a light with nothing to draw.
    std::vector<shading::Material>  materials = scene.materials;
    std::vector<Volume_light_gpu>   volume_lights;
    std::vector<Emission_dist_host> dists;
    for (Instance_desc const& in : scene.instances) {
        if (!in.light) {
            continue;
        }
        std::vector<uint32_t> slots = scene.meshes[in.mesh].tri_slot;
        std::sort(slots.begin(), slots.end());
        slots.erase(std::unique(slots.begin(), slots.end()), slots.end());
        for (uint32_t const slot : slots) {
            uint32_t const     mat = material_of(in, slot);
            shading::Material& m   = materials[mat];
            if (m.type != shading::Type_volume || !(m.emission.x > 0.f || m.emission.y > 0.f || m.emission.z > 0.f)) {
                continue;
            }
            if (m.volume_light != 0) {
                error_ = "an emitting medium's material lights more than one prop (each needs its own)";
                return SPB_ERROR_ARGUMENT;
            }
            m.volume_light = shading::Volume_light_unsampled;
            if (!in.cube) {
                continue;
            }
            float const*     t = in.trafo;
            Volume_light_gpu vl{};
            vl.m0 = make_float4(t[0], t[4], t[8], t[12]);
            vl.m1 = make_float4(t[1], t[5], t[9], t[13]);
            vl.m2 = make_float4(t[2], t[6], t[10], t[14]);
            // Cube::volume (cube.cpp:229-232): the cube [-1, 1]^3 scaled
            double const det = double(t[0]) * (double(t[5]) * t[10] - double(t[6]) * t[9]) -
                               double(t[1]) * (double(t[4]) * t[10] - double(t[6]) * t[8]) +
                               double(t[2]) * (double(t[4]) * t[9] - double(t[5]) * t[8]);
            double const volume = 8.0 * std::fabs(det);
            vl.volume           = float(volume);
            vl.material         = mat;
            // the average radiance its power is taken from (volumetric::Material::prepare_sampling,
            // volumetric_material.cpp:40-44, or the grid's mean of density x emission)
            double average[3] = {double(m.mu_a.x) * m.emission.x, double(m.mu_a.y) * m.emission.y,
                                 double(m.mu_a.z) * m.emission.z};
            if (m.medium != 0 && scene.media[m.medium - 1].color[0] != 0) {
                // a colour grid: uniform points (a Volume light, not an image), its power from
                // the material's default coefficients of 0.5 (Grid_color's cc_,
                // volumetric_grid.cpp:320-324, through Material::prepare_sampling)
                vl.medium = m.medium - 1;
                vl.color  = 1;
                for (int k = 0; k < 3; ++k) {
                    average[k] = 0.5 * double((&m.emission.x)[k]);
                }
            } else if (m.medium != 0) {
                Grid_medium const& gm = scene.media[m.medium - 1];
                double const       maj_a = std::max({double(m.mu_a.x), double(m.mu_a.y), double(m.mu_a.z)});
                if (!(maj_a > 0.0)) {
                    continue;  // a medium that absorbs nothing emits nothing
                }
                std::vector<float4> table(16);
                for (int k = 0; k < 16; ++k) {
                    table[k] = make_float4(gm.blackbody[3 * k], gm.blackbody[3 * k + 1], gm.blackbody[3 * k + 2], 0.f);
                }
                bool const         hot = gm.temperature != 0;
                Emission_dist_host d   = emission_distribution(
                    scene.grids[gm.grid], m.emission, hot ? scene.grids[gm.temperature - 1].density : nullptr,
                    hot ? table.data() : nullptr,
                    gm.emission_scale != 0 ? scene.grids[gm.emission_scale - 1].density : nullptr);
                if (!(d.total > 0.0)) {
                    continue;
                }
                d.repeat            = gm.repeat;
                double const voxels = double(d.dims[0]) * d.dims[1] * d.dims[2];
                vl.medium           = m.medium - 1;
                vl.dist             = uint32_t(dists.size()) + 1;
                vl.pdf_factor       = float(voxels / maj_a);
                vl.a_norm = v3(m.mu_a.x > 0.f ? float(maj_a / m.mu_a.x) : 0.f, m.mu_a.y > 0.f ? float(maj_a / m.mu_a.y) : 0.f,
                               m.mu_a.z > 0.f ? float(maj_a / m.mu_a.z) : 0.f);
                std::copy(d.average, d.average + 3, average);
                dists.push_back(std::move(d));
            }
            Light_input li;
            for (int k = 0; k < 3; ++k) {
                li.a[k] = 1e300;
                li.b[k] = -1e300;
            }
            for (int c = 0; c < 8; ++c) {
                double const o[3] = {c & 1 ? 1.0 : -1.0, c & 2 ? 1.0 : -1.0, c & 4 ? 1.0 : -1.0};
                for (int k = 0; k < 3; ++k) {
                    double const w = o[0] * t[k] + o[1] * t[4 + k] + o[2] * t[8 + k] + t[12 + k];
                    li.a[k]        = std::min(li.a[k], w);
                    li.b[k]        = std::max(li.b[k], w);
                }
            }
            for (int k = 0; k < 3; ++k) {
                li.c[k] = 0.5 * (li.a[k] + li.b[k]);
            }
            li.volume    = uint32_t(volume_lights.size()) + 1;
            li.power     = volume * std::max({average[0], average[1], average[2]});
            li.two_sided = true;
            li.slot      = light_slots + uint32_t(volume_lights.size());
            li.material  = mat;
            if (volume > 0.0 && li.power > 0.0) {
                emitters.push_back(li);
                volume_lights.push_back(vl);
            }
        }
    }

    Light_tree tree;
    build_light_tree(emitters, std::max(light_slots + uint32_t(volume_lights.size()), 1u), tree);
    d_->num_lights = tree.num_lights;
    for (size_t k = 0; k < volume_lights.size(); ++k) {
        materials[volume_lights[k].material].volume_light = tree.order[light_slots + k] + 1;
    }

    // Scene box for the guide's position encoding; a new scene starts a new guide.
    {
        d_->bounds_lo  = make_float4(float(lo[0]), float(lo[1]), float(lo[2]), 0.f);
        d_->bounds_inv = make_float4(1.f / std::max(float(hi[0] - lo[0]), 1e-6f), 1.f / std::max(float(hi[1] - lo[1]), 1e-6f),
                                     1.f / std::max(float(hi[2] - lo[2]), 1e-6f), 0.f);
        d_->net_ready  = false;
    }

    // The environment's share of light picks: its power against the emitters', with the
    // reference's power of an infinite light, squared scene extent x 4 pi x the largest radiance
    // component (Light::power, light.cpp:38-48; Tree_builder, light_tree_builder.cpp:527-537).
    float const* env = scene.environment;
    d_->env          = make_float4(env[0], env[1], env[2], 0.f);
    if (scene.environment_light && (env[0] > 0.f || env[1] > 0.f || env[2] > 0.f)) {
        double ext2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            ext2 += (hi[k] - lo[k]) * (hi[k] - lo[k]);
        }
        double const p_env = ext2 * 4.0 * 3.14159265358979323846 *
                             std::max({double(env[0]), double(env[1]), double(env[2])});
        double p_finite = 0.0;
        for (Light_input const& li : emitters) {
            p_finite += li.power;
        }
        d_->env.w = float(p_env / (p_env + p_finite));
    }
    // Split light selection: the depth the split walk starts at, so that the environment and
    // the most emitters one walk can return fit Max_light_picks (Tree_builder,
    // light_tree_builder.cpp:510-522), and that most.
    {
        uint32_t const infinite = d_->env.w > 0.f ? 1u : 0u;
        uint32_t       bias     = 0;
        if (infinite != 0 && tree.num_nodes != 0) {
            uint32_t const left = Max_light_picks - max_split_picks(tree, 0);
            if (left < infinite) {
                bias = std::max(uint32_t(std::ceil(std::log2(double(infinite - left)))), 1u);
            }
        }
        d_->split_depth_bias = bias;
        d_->max_picks        = (tree.num_nodes != 0 ? max_split_picks(tree, bias) : 0u) + infinite;
    }

    SPB_RCUDA(upload(d_->tri_info, info.data(), info.size() * sizeof(uint4)));
    SPB_RCUDA(upload(d_->positions, pos.data(), pos.size() * sizeof(float4)));
    SPB_RCUDA(upload(d_->normals, nrm.data(), nrm.size() * sizeof(float4)));
    SPB_RCUDA(upload(d_->uvs, uv.data(), uv.size() * sizeof(float2)));
    // Material textures, each as float4 texels.
    for (float4*& t : d_->texture_texels) {
        free_ptr(t);
    }
    d_->texture_texels.assign(scene.textures.size(), nullptr);
    std::vector<Texture_gpu> tex_table(scene.textures.size());
    for (size_t k = 0; k < scene.textures.size(); ++k) {
        Texture_desc const& td = scene.textures[k];
        size_t const        n  = size_t(td.width) * td.height;
        if (td.channels < 1 || td.channels > 4 || td.texels.size() != n * td.channels) {
            error_ = "texture with inconsistent texels";
            return SPB_ERROR_ARGUMENT;
        }
        std::vector<float4> texels(n, make_float4(0.f, 0.f, 0.f, 0.f));
        for (size_t i = 0; i < n; ++i) {
            float v[4] = {0.f, 0.f, 0.f, 0.f};
            for (uint32_t c = 0; c < td.channels; ++c) {
                v[c] = td.texels[i * td.channels + c];
            }
            texels[i] = make_float4(v[0], v[1], v[2], v[3]);
        }
        SPB_RCUDA(upload(d_->texture_texels[k], texels.data(), texels.size() * sizeof(float4)));
        tex_table[k] = Texture_gpu{d_->texture_texels[k], int(td.width), int(td.height),
                                   (td.nearest ? 1u : 0u) | (td.clamp ? 2u : 0u), td.scale[0], td.scale[1], {0, 0}};
    }
    free_ptr(d_->textures);
    if (!tex_table.empty()) {
        SPB_RCUDA(upload(d_->textures, tex_table.data(), tex_table.size() * sizeof(Texture_gpu)));
    }
    SPB_RCUDA(upload(d_->materials, materials.data(), materials.size() * sizeof(shading::Material)));
    SPB_RCUDA(upload(d_->light_nodes, tree.nodes.data(), tree.nodes.size() * sizeof(float)));
    d_->light_tree_nodes      = tree.nodes;
    d_->split_radii_threshold = -1.f;  // split radii set at the first render
    SPB_RCUDA(upload(d_->light_cones, tree.cones.data(), tree.cones.size() * sizeof(float)));
    SPB_RCUDA(upload(d_->light_tris, tree.tris.data(), tree.tris.size() * sizeof(float)));
    SPB_RCUDA(upload(d_->light_order, tree.order.data(), tree.order.size() * sizeof(uint32_t)));
    SPB_RCUDA(upload(d_->e_table, ggx_albedo_table(),
                     Ggx_table_size * Ggx_table_size * sizeof(float)));

    // Density grids and the media that sample them.
    free_grids();
    std::vector<Medium_gpu> media;
    for (Density_grid const& g : scene.grids) {
        size_t const n = size_t(g.dims[0]) * g.dims[1] * g.dims[2];
        d_->grid_density.push_back(nullptr);
        SPB_RCUDA(upload(d_->grid_density.back(), g.density, n * sizeof(float)));
    }
    d_->grid_cells.assign(scene.media.size(), nullptr);
    std::vector<float4> tables(16 * std::max<size_t>(scene.media.size(), 1));
    for (size_t k = 0; k < scene.media.size(); ++k) {
        for (int i = 0; i < 16; ++i) {
            float const* b    = scene.media[k].blackbody + 3 * i;
            tables[16 * k + i] = make_float4(b[0], b[1], b[2], 0.f);
        }
    }
    SPB_RCUDA(upload(d_->blackbody, tables.data(), tables.size() * sizeof(float4)));
    for (size_t k = 0; k < scene.media.size(); ++k) {
        Grid_medium const& gm = scene.media[k];
        if (gm.grid >= scene.grids.size() || gm.temperature > scene.grids.size() ||
            gm.emission_scale > scene.grids.size()) {
            error_ = "medium refers to a missing density grid";
            return SPB_ERROR_ARGUMENT;
        }
        if (gm.emission_scale != 0 && !std::equal(scene.grids[gm.grid].dims, scene.grids[gm.grid].dims + 3,
                                                  scene.grids[gm.emission_scale - 1].dims)) {
            error_ = "an emission-scale grid must have its density grid's dimensions";
            return SPB_ERROR_ARGUMENT;
        }
        if (gm.temperature != 0 &&
            !std::equal(scene.grids[gm.grid].dims, scene.grids[gm.grid].dims + 3, scene.grids[gm.temperature - 1].dims)) {
            error_ = "a temperature grid must have its density grid's dimensions";
            return SPB_ERROR_ARGUMENT;
        }
        Density_grid const& g = scene.grids[gm.grid];
        Medium_gpu          mg{};
        float const*        r = gm.world_to_uvw;
        mg.m0      = make_float4(r[0], r[1], r[2], r[3]);
        mg.m1      = make_float4(r[4], r[5], r[6], r[7]);
        mg.m2      = make_float4(r[8], r[9], r[10], r[11]);
        mg.density = d_->grid_density[gm.grid];
        mg.nx      = int(g.dims[0]);
        mg.ny      = int(g.dims[1]);
        mg.nz      = int(g.dims[2]);
        int const cells[3] = {(mg.nx + (1 << Cell_log2) - 1) >> Cell_log2,
                              (mg.ny + (1 << Cell_log2) - 1) >> Cell_log2,
                              (mg.nz + (1 << Cell_log2) - 1) >> Cell_log2};
        mg.cx    = cells[0];
        mg.cy    = cells[1];
        mg.cz    = cells[2];
        mg.flags = (gm.nearest ? 1u : 0u) | (gm.repeat ? 2u : 0u);
        if (gm.temperature != 0) {
            mg.temperature = d_->grid_density[gm.temperature - 1];
            mg.blackbody   = d_->blackbody + 16 * k;
        }
        if (gm.emission_scale != 0) {
            mg.scale = d_->grid_density[gm.emission_scale - 1];
        }
        if (gm.color[0] != 0) {
            for (int c = 0; c < 3; ++c) {
                if (gm.color[c] == 0 || gm.color[c] > scene.grids.size() ||
                    !std::equal(scene.grids[gm.grid].dims, scene.grids[gm.grid].dims + 3,
                                scene.grids[gm.color[c] - 1].dims)) {
                    error_ = "a colour grid's channels must share its dimensions";
                    return SPB_ERROR_ARGUMENT;
                }
                mg.rgb[c] = d_->grid_density[gm.color[c] - 1];
            }
            mg.color_distance = gm.color_distance;
            mg.color_maj      = -std::log(0.01f) / gm.color_distance;
        }
        int const num_cells = cells[0] * cells[1] * cells[2];
        free_ptr(d_->grid_cells[k]);
        SPB_RCUDA(dev_malloc(&d_->grid_cells[k], size_t(num_cells) * sizeof(float2)));
        k_majorant_cells<<<(num_cells + 127) / 128, 128, 0, d_->stream>>>(mg.density, mg.nx, mg.ny, mg.nz, cells[0],
                                                                          cells[1], cells[2], gm.repeat,
                                                                          d_->grid_cells[k]);
        SPB_RCUDA(cudaGetLastError());
        SPB_RCUDA(cudaStreamSynchronize(d_->stream));
        mg.cells = d_->grid_cells[k];
        media.push_back(mg);
    }
    SPB_RCUDA(upload(d_->media, media.data(), media.size() * sizeof(Medium_gpu)));
    // Emitting media that are lights, and the emission distributions of their grids.
    std::vector<Emission_dist_gpu> dist_table;
    for (Emission_dist_host const& d : dists) {
        d_->dist_data.push_back(nullptr);
        SPB_RCUDA(upload(d_->dist_data.back(), d.data.data(), d.data.size() * sizeof(float)));
        size_t const      n = size_t(d.dims[0]) * d.dims[1] * d.dims[2];
        Emission_dist_gpu e{};
        e.prob   = d_->dist_data.back();
        e.cdf_z  = e.prob + n;
        e.cdf_y  = e.cdf_z + (d.dims[2] + 1);
        e.cdf_x  = e.cdf_y + size_t(d.dims[2]) * (d.dims[1] + 1);
        e.nx     = int(d.dims[0]);
        e.ny     = int(d.dims[1]);
        e.nz     = int(d.dims[2]);
        e.repeat = d.repeat ? 1u : 0u;
        dist_table.push_back(e);
    }
    SPB_RCUDA(upload(d_->emission_dists, dist_table.data(), dist_table.size() * sizeof(Emission_dist_gpu)));
    SPB_RCUDA(upload(d_->volume_lights, volume_lights.data(), volume_lights.size() * sizeof(Volume_light_gpu)));
    scene_ready_ = true;
    return SPB_OK;
}

int32_t Renderer::set_camera(Camera_desc const& camera) {
    return set_views(std::vector<Camera_desc>{camera});
}

int32_t Renderer::set_views(std::vector<Camera_desc> const& views) {
    clear_graphs();
    if (views.empty() || views.size() > Max_views) {
        error_ = "between 1 and " + std::to_string(Max_views) + " views";
        return SPB_ERROR_ARGUMENT;
    }
    std::vector<Cam>      cams(views.size());
    std::vector<uint32_t> traced(views.size() + 1, 0), film(views.size() + 1, 0);
    for (size_t v = 0; v < views.size(); ++v) {
        Camera_desc const& c = views[v];
        if (c.width == 0 || c.height == 0 || !(c.fov > 0.f) || c.width > 65536 || c.height > 65536) {
            error_ = "camera needs a resolution and a field of view";
            return SPB_ERROR_ARGUMENT;
        }
        // Perspective::on_update (camera_perspective.cpp:203-224): image plane at distance
        // 1 / tan(fov / 2), x in [-1, 1], y in [-h/w, h/w]
        float const ratio = float(c.height) / float(c.width);
        float const z     = 1.f / std::tan(0.5f * c.fov);
        Cam&        cam   = cams[v];
        cam.left_top      = make_float3(-1.f, ratio, z);
        cam.d_x           = make_float3(2.f / float(c.width), 0.f, 0.f);
        cam.d_y           = make_float3(0.f, -2.f * ratio / float(c.height), 0.f);
        cam.r0            = make_float3(c.rotation[0], c.rotation[1], c.rotation[2]);
        cam.r1            = make_float3(c.rotation[3], c.rotation[4], c.rotation[5]);
        cam.r2            = make_float3(c.rotation[6], c.rotation[7], c.rotation[8]);
        cam.pos           = make_float3(c.position[0], c.position[1], c.position[2]);
        cam.w             = c.width;
        cam.h             = c.height;
        uint64_t const t  = uint64_t(traced[v]) + uint64_t(c.width + 2 * Film_border) * (c.height + 2 * Film_border);
        uint64_t const f  = uint64_t(film[v]) + uint64_t(c.width) * c.height;
        if (t >= (1ull << 31)) {
            error_ = "views too large";
            return SPB_ERROR_ARGUMENT;
        }
        traced[v + 1] = uint32_t(t);
        film[v + 1]   = uint32_t(f);
    }
    views_ = views;
    SPB_RCUDA(upload(d_->cams, cams.data(), cams.size() * sizeof(Cam)));
    SPB_RCUDA(upload(d_->view_offsets, traced.data(), traced.size() * sizeof(uint32_t)));
    SPB_RCUDA(upload(d_->film_offsets, film.data(), film.size() * sizeof(uint32_t)));
    d_->num_views     = uint32_t(views.size());
    d_->traced_pixels = traced.back();
    uint32_t const pixels = film.back();
    if (pixels != d_->film_pixels) {
        free_ptr(d_->film);
        free_ptr(d_->comp);
        free_ptr(d_->out);
        SPB_RCUDA(dev_malloc(&d_->film, pixels * sizeof(float4)));
        SPB_RCUDA(dev_malloc(&d_->comp, pixels * sizeof(float4)));
        SPB_RCUDA(dev_malloc(&d_->out, pixels * sizeof(float4)));
        d_->film_pixels = pixels;
    }
    camera_ready_ = true;
    return start_frame();
}

int32_t Renderer::start_frame() {
    if (!d_->film) {
        error_ = "no camera";
        return SPB_ERROR_STATE;
    }
    SPB_RCUDA(cudaMemsetAsync(d_->film, 0, d_->film_pixels * sizeof(float4), d_->stream));
    SPB_RCUDA(cudaMemsetAsync(d_->comp, 0, d_->film_pixels * sizeof(float4), d_->stream));
    return SPB_OK;
}

int32_t Renderer::ensure_buffers(uint32_t paths, uint32_t picks_per_path) {
    uint64_t const picks = uint64_t(paths) * picks_per_path;
    if (paths <= d_->capacity && picks <= d_->pick_capacity) {
        return SPB_OK;
    }
    clear_graphs();
    Paths& p = d_->paths;
    free_ptr(p.ray_o);
    free_ptr(p.ray_d);
    free_ptr(p.hit_id);
    free_ptr(p.hit_inst);
    free_ptr(p.hit_t);
    free_ptr(p.hit_uv);
    free_ptr(p.T);
    free_ptr(p.L);
    free_ptr(p.puv);
    free_ptr(p.rng);
    free_ptr(p.info);
    free_ptr(p.sh_o);
    free_ptr(p.sh_d);
    free_ptr(p.sh_L);
    free_ptr(p.prev_n);
    free_ptr(p.split_o);
    free_ptr(p.sh2_o);
    free_ptr(p.sh2_d);
    free_ptr(p.sh2_L);
    free_ptr(p.split_m);
    free_ptr(p.pick_d);
    free_ptr(p.pick_c);
    free_ptr(p.L2);
    free_ptr(p.guide_in);
    free_ptr(p.guide_out);
    free_ptr(p.guide_ok);
    free_ptr(p.rec);
    free_ptr(p.open_record);
    d_->guide_paths = 0;
    free_ptr(d_->queue[0]);
    free_ptr(d_->queue[1]);
    free_ptr(d_->shadow_queue);
    free_ptr(d_->transmit_queue);
    free_ptr(d_->transmit_pick_queue);
    size_t const n = paths;
    SPB_RCUDA(dev_malloc(&p.ray_o, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.ray_d, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.hit_id, n * sizeof(uint32_t)));
    SPB_RCUDA(dev_malloc(&p.hit_inst, n * sizeof(uint32_t)));
    SPB_RCUDA(dev_malloc(&p.hit_t, n * sizeof(float)));
    SPB_RCUDA(dev_malloc(&p.hit_uv, n * sizeof(float2)));
    SPB_RCUDA(dev_malloc(&p.T, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.L, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.puv, n * sizeof(float2)));
    SPB_RCUDA(dev_malloc(&p.rng, n * sizeof(uint4)));
    SPB_RCUDA(dev_malloc(&p.info, n * sizeof(uint32_t)));
    SPB_RCUDA(dev_malloc(&p.sh_o, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.sh_d, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.sh_L, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.sh2_o, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.sh2_d, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.sh2_L, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.prev_n, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.L2, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&d_->queue[0], n * sizeof(uint32_t)));
    SPB_RCUDA(dev_malloc(&d_->queue[1], n * sizeof(uint32_t)));
    // Split selections: a record per path and every light its selection can return.  Shadow
    // rays: a path's two slots and every pick.
    size_t const np = std::max<size_t>(size_t(n) * picks_per_path, 1);
    SPB_RCUDA(dev_malloc(&p.split_o, n * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.split_m, n * sizeof(uint4)));
    SPB_RCUDA(dev_malloc(&p.pick_d, np * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&p.pick_c, np * sizeof(float4)));
    SPB_RCUDA(dev_malloc(&d_->shadow_queue, (2 * n + np) * sizeof(uint32_t)));
    SPB_RCUDA(dev_malloc(&d_->transmit_queue, 2 * n * sizeof(uint32_t)));
    SPB_RCUDA(dev_malloc(&d_->transmit_pick_queue, np * sizeof(uint32_t)));
    d_->pick_capacity = uint64_t(n) * picks_per_path;
    if (!d_->counters) {
        SPB_RCUDA(dev_malloc(&d_->counters, Counter_words * sizeof(uint32_t)));
    }
    d_->capacity = paths;
    return SPB_OK;
}

// Guide buffers for `paths` paths: network outputs, validity, training records; the training
// batch arrays; the network itself (initialised once per scene).
int32_t Renderer::ensure_guide(uint32_t paths) {
    Paths&         p  = d_->paths;
    uint32_t const rd = settings_.record_depth;
    if (d_->guide_paths < paths || d_->guide_records != rd) {
        clear_graphs();
        free_ptr(p.guide_in);
        free_ptr(p.guide_out);
        free_ptr(p.guide_ok);
        free_ptr(p.rec);
        free_ptr(p.open_record);
        size_t const n = d_->capacity;
        size_t const tiled_entries = (n + guide::Tile - 1) / guide::Tile * guide::Tile;
        SPB_RCUDA(dev_malloc(&p.guide_in, tiled_entries * guide::Inputs * sizeof(__nv_bfloat16)));
        SPB_RCUDA(dev_malloc(&p.guide_out, n * Mixture_floats * sizeof(float)));
        SPB_RCUDA(dev_malloc(&p.guide_ok, n));
        SPB_RCUDA(dev_malloc(&p.rec, n * rd * Record_float4 * sizeof(float4)));
        SPB_RCUDA(dev_malloc(&p.open_record, n * sizeof(uint32_t)));
        d_->guide_paths   = uint32_t(n);
        d_->guide_records = rd;
    }
    uint32_t const batch = settings_.guide_batch;
    if (d_->train_capacity < batch) {
        free_ptr(d_->train_in);
        free_ptr(d_->train_dir);
        free_ptr(d_->train_w);
        free_ptr(d_->train_parts);
        size_t const rows = (size_t(batch) + guide::Tile - 1) / guide::Tile * guide::Tile;
        SPB_RCUDA(dev_malloc(&d_->train_in, rows * guide::Inputs * sizeof(__nv_bfloat16)));
        SPB_RCUDA(dev_malloc(&d_->train_dir, size_t(batch) * 3 * sizeof(float)));
        SPB_RCUDA(dev_malloc(&d_->train_w, size_t(batch) * sizeof(float)));
        SPB_RCUDA(dev_malloc(&d_->train_parts, (rows + 255) / 256 * sizeof(float)));
        d_->train_capacity = batch;
        clear_graphs();
        SPB_RCUDA(cudaError_t(d_->net.prepare_gradients(batch)));
    }
    if (!d_->pass_counter) {
        SPB_RCUDA(dev_malloc(&d_->pass_counter, sizeof(uint32_t)));
        d_->net_ready = false;
    }
    if (!d_->net_ready) {
        clear_graphs();
        SPB_RCUDA(cudaError_t(d_->net.init(settings_.guide_seed)));
        SPB_RCUDA(cudaFuncSetAttribute(k_guide, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(sizeof(Infer_smem))));
        // Persistent inference: as many blocks as fit on the SMs at once, from the SM's shared
        // memory and registers (the blocks are independent, so any count is correct).
        SPB_RCUDA(cudaFuncSetAttribute(k_guide, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       int(cudaSharedmemCarveoutMaxShared)));
        int dev = 0, sms = 0, smem_sm = 0, reserved = 0, regs_sm = 0;
        SPB_RCUDA(cudaGetDevice(&dev));
        SPB_RCUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        SPB_RCUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        SPB_RCUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
        SPB_RCUDA(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
        cudaFuncAttributes fa{};
        SPB_RCUDA(cudaFuncGetAttributes(&fa, k_guide));
        int const warp_regs = (fa.numRegs * 32 + 255) / 256 * 256;  // allocated per warp in 256s
        int const per_sm    = std::min({smem_sm / (int(sizeof(Infer_smem)) + reserved),
                                        regs_sm / std::max(1, warp_regs * (guide::Block / 32)), 2048 / guide::Block});
        d_->guide_grid = uint32_t(std::max(1, sms * std::max(1, per_sm)));
        SPB_RCUDA(cudaMemset(d_->pass_counter, 0, sizeof(uint32_t)));
        d_->net_ready = true;
    }
    return SPB_OK;
}

// Drops the captured wave graphs (their kernels hold buffer and scene pointers).
void Renderer::clear_graphs() {
    for (auto const& g : d_->graphs) {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
        }
    }
    d_->graphs.clear();
    if (d_->train_graph.exec) {
        cudaGraphExecDestroy(d_->train_graph.exec);
    }
    d_->train_graph = Device::Train_graph{0, 0, 0, 0.f, nullptr};
}

// Training after a pass: guide_steps Adam steps, each on a fresh batch of the pass's records.
// The batch counter and Adam's step count live in device memory, so a pass of a recurring shape
// is captured once as a graph and replayed (no host launch gaps between its ~100 launches).
int32_t Renderer::train_guide(uint32_t paths) {
    cudaStream_t   st      = d_->stream;
    uint32_t const batch   = settings_.guide_batch;
    uint32_t const records = paths * settings_.record_depth;
    uint32_t const steps   = settings_.guide_steps;
    float const    lr      = settings_.guide_lr;
    // one thread per batch row, the last tile's rows past the batch included
    uint32_t const gather_blocks = ((batch + guide::Tile - 1) / guide::Tile * guide::Tile + 255) / 256;
    auto const     enqueue_pass  = [&]() -> int32_t {
        for (uint32_t step = 0; step < steps; ++step) {
            k_train_gather<<<gather_blocks, 256, 0, st>>>(d_->paths, d_->launch_dev, records, batch, d_->pass_counter,
                                                          d_->train_in, d_->train_dir, d_->train_w, d_->train_parts);
            SPB_RCUDA(cudaError_t(d_->net.gradients_tiled(d_->train_in, d_->train_dir, d_->train_w, batch,
                                                          d_->train_parts, gather_blocks, st)));
            SPB_RCUDA(cudaError_t(d_->net.adam_counted(lr, d_->pass_counter, st)));
        }
        return SPB_OK;
    };
    if (!settings_.cuda_graphs) {
        return enqueue_pass();
    }
    Device::Train_graph& g = d_->train_graph;
    if (!g.exec || g.records != records || g.batch != batch || g.steps != steps || g.lr != lr) {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
        SPB_RCUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int32_t const     e     = enqueue_pass();
        cudaGraph_t       graph = nullptr;
        cudaError_t const ce    = cudaStreamEndCapture(st, &graph);
        if (e != SPB_OK || ce != cudaSuccess) {
            if (graph) {
                cudaGraphDestroy(graph);
            }
            return e != SPB_OK ? e : fail_cuda("cudaStreamEndCapture", int(ce));
        }
        cudaGraphExec_t   exec = nullptr;
        cudaError_t const ie   = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        SPB_RCUDA(ie);
        g = Device::Train_graph{records, batch, steps, lr, exec};
    }
    SPB_RCUDA(cudaGraphLaunch(g.exec, st));
    return SPB_OK;
}

// Squared distance from a light-tree node's centre beyond which split_node cannot pass for
// the splitting measure S = (1 / t - 1)^2, or 0 if it passes nowhere.  The test is g >= 0 for
// g = (ve + ee^2) (b - a)^2 + 3 ve a b - 3 S (a b)^3 with a = max(d - r, E), b = d + r, E = 0.001.
// Beyond d = r + E, in x = d^2 - r^2, g = 4 r^2 (ve + ee^2) + 3 ve x - 3 S x^3 is concave, so it
// is negative beyond its largest root, found by bisection.  Below (a = E, b = d + r in
// [r, 2 r + E]) g is a cubic in b whose maximum lies at an end or a critical point; when that
// maximum is clearly negative the node never splits.  The radius is widened by 1 % so that the
// float test on the device never passes beyond it.
static float split_radius2(double r, double ve, double vee, double S) {
    if (S <= 0.0) {
        return INFINITY;
    }
    double const E  = 0.001;
    auto const   g2 = [&](double x) { return 4.0 * r * r * vee + 3.0 * ve * x - 3.0 * S * x * x * x; };
    double const x0 = (r + E) * (r + E) - r * r;
    double const xs = std::max(x0, ve > 0.0 ? std::sqrt(ve / (3.0 * S)) : x0);
    double       dmax;
    if (g2(xs) >= 0.0) {
        double lo = xs, hi = std::max(2.0 * xs, 1e-12);
        while (g2(hi) >= 0.0 && hi < 1e30) {
            lo = hi;
            hi *= 2.0;
        }
        for (int i = 0; i < 100; ++i) {
            double const mid = 0.5 * (lo + hi);
            (g2(mid) >= 0.0 ? lo : hi) = mid;
        }
        dmax = std::sqrt(hi + r * r);
    } else {
        auto const G = [&](double b) {
            double const eb = E * b;
            return vee * (b - E) * (b - E) + 3.0 * ve * eb - 3.0 * S * eb * eb * eb;
        };
        double       gmax = std::max(G(r), G(2.0 * r + E));
        double const A    = 9.0 * S * E * E * E, B = -2.0 * vee, C = 2.0 * vee * E - 3.0 * ve * E;
        double const disc = B * B - 4.0 * A * C;
        if (disc >= 0.0) {
            for (double const sgn : {1.0, -1.0}) {
                double const b = (-B + sgn * std::sqrt(disc)) / (2.0 * A);
                if (b >= r && b <= 2.0 * r + E) {
                    gmax = std::max(gmax, G(b));
                }
            }
        }
        double const b1    = 2.0 * r + E;
        double const scale = std::max({std::fabs(vee * 4.0 * r * r), std::fabs(3.0 * ve * E * b1),
                                       std::fabs(3.0 * S * E * E * E * b1 * b1 * b1), 1e-300});
        if (gmax < -1e-4 * scale) {
            return 0.f;
        }
        dmax = r + E;
    }
    double const d = 1.01 * dmax + 1e-6;
    return float(d * d);
}

int32_t Renderer::render(uint32_t first_sample, uint32_t num_samples) {
    if (!ready()) {
        error_ = "render needs a scene and a camera";
        return SPB_ERROR_STATE;
    }
    if (!d_->pinned_count) {
        error_ = "no pinned host memory (CUDA unavailable)";
        return SPB_ERROR_CUDA;
    }
    if (settings_.max_bounces + 2 > Max_bounce_slots) {
        error_ = "max_bounces too large";
        return SPB_ERROR_ARGUMENT;
    }
    // camera samples per sample slot: the image and its filter border
    uint32_t const pixels = d_->traced_pixels;
    // Wave size: k samples per pixel per wave, k = paths per wave / pixels (at least 1), the
    // paths per wave from the settings or the autotuner; buffers hold the largest candidate.
    bool const     tuning     = settings_.wave_paths == 0 || settings_.trace_blocks_per_sm == 0;
    // Split light selection: every path of a wave may select up to max_picks lights; waves are
    // bounded so that their picks fit Pick_budget bytes.
    uint32_t const picks_per_path = settings_.light_split && d_->max_picks > 1 ? d_->max_picks : 0u;
    uint32_t const pick_paths =
        picks_per_path ? uint32_t(std::min<uint64_t>(Tuner::Max_wave_paths,
                                                      Pick_budget / (uint64_t(picks_per_path) * 2 * sizeof(float4))))
                       : Tuner::Max_wave_paths;
    uint32_t const max_paths =
        std::min(settings_.wave_paths ? settings_.wave_paths : Tuner::Max_wave_paths, pick_paths);
    auto const     wave_spp   = [&](uint32_t paths_per_wave) {
        return std::max(1u, std::min(num_samples, paths_per_wave / std::max(1u, pixels)));
    };
    uint32_t const max_wave = wave_spp(max_paths);
    // while the guide trains, passes of guide_pass_spp with training steps in between
    uint32_t const train_wave = std::max(1u, std::min(max_wave, settings_.guide_pass_spp));
    // Golden ratio sequences over the frame's samples (first_sample + num_samples per pixel).
    uint32_t const golden_n = settings_.golden_ratio ? first_sample + num_samples : 0u;
    if (golden_n != 0 && golden_n != d_->golden_n) {
        std::vector<uint32_t> sorted(golden_n);
        for (uint32_t j = 0; j < golden_n; ++j) {
            sorted[j] = j * 2654435769u;
        }
        std::sort(sorted.begin(), sorted.end());
        SPB_RCUDA(upload(d_->golden_sorted, sorted.data(), sorted.size() * sizeof(uint32_t)));
        d_->golden_n = golden_n;
    }
    if (settings_.light_split && d_->split_radii_threshold != settings_.split_threshold &&
        !d_->light_tree_nodes.empty()) {
        double const t = settings_.split_threshold;
        double const S = t >= 1.0 ? 0.0 : (1.0 / t - 1.0) * (1.0 / t - 1.0);
        std::vector<float>& nodes = d_->light_tree_nodes;
        for (size_t n = 0; n + Light_node_floats <= nodes.size(); n += Light_node_floats) {
            nodes[n + 15] = split_radius2(nodes[n + 3], nodes[n + 12], nodes[n + 14], S);
        }
        SPB_RCUDA(cudaMemcpy(d_->light_nodes, nodes.data(), nodes.size() * sizeof(float), cudaMemcpyHostToDevice));
        d_->split_radii_threshold = settings_.split_threshold;
    }
    if (settings_.spectral) {
        // the persistent spectral kernel keeps its paths in registers: no wave buffers; its
        // guiding is the phase guide at medium vertices
        if (!d_->spectral_scene || d_->instanced) {
            error_ = "spectral rendering takes scenes of homogeneous or density-grid media (not emitting), "
                     "emitters and the environment, in one tree";
            return SPB_ERROR_ARGUMENT;
        }
        if (!d_->counters) {
            SPB_RCUDA(dev_malloc(&d_->counters, Counter_words * sizeof(uint32_t)));
        }
    } else if (int32_t const st = ensure_buffers(max_wave * pixels, picks_per_path)) {
        return st;
    }
    if (settings_.guiding && !settings_.spectral) {
        if (int32_t const st = ensure_guide(max_wave * pixels)) {
            return st;
        }
    }

    Scene_gpu sg;
    sg.nodes         = d_->nodes;
    sg.tris          = d_->tris;
    sg.hit_margin    = d_->hit_margin;
    sg.tri_info      = d_->tri_info;
    sg.positions     = d_->positions;
    sg.normals       = d_->normals;
    sg.materials     = d_->materials;
    sg.light_nodes   = d_->light_nodes;
    sg.light_cones   = d_->light_cones;
    sg.light_tris    = d_->light_tris;
    sg.light_order   = d_->light_order;
    sg.num_lights    = d_->num_lights;
    sg.env           = d_->env;
    sg.e_table       = d_->e_table;
    sg.media         = d_->media;
    sg.volume_lights  = d_->volume_lights;
    sg.emission_dists = d_->emission_dists;
    sg.inst_trace     = d_->inst_trace;
    sg.inst_shade     = d_->inst_shade;
    sg.inst_materials = d_->inst_materials;
    sg.instanced      = d_->instanced ? 1u : 0u;
    sg.tracking_capped = d_->counters + Overflow_slot + 2;
    sg.split_bounces    = settings_.light_split ? Split_bounces : 0u;
    sg.split_depth_bias = d_->split_depth_bias;
    {
        // t >= 1 splits every node the walk passes above Max_split_depth
        double const t = settings_.split_threshold;
        sg.split_scale = t >= 1.0 ? 0.f : float(3.0 * (1.0 / t - 1.0) * (1.0 / t - 1.0));
    }
    sg.uvs             = d_->uvs;
    sg.textures        = d_->textures;

    cudaStream_t const st = d_->stream;
    uint32_t* const    ctr = d_->counters;
    // One iteration per path vertex.  Medium boundaries are null vertices: they take an
    // iteration without counting as a bounce (Straight_transmission keeps ray.depth,
    // pathtracer_mis.cpp:180-182), so with media the loop goes on while paths remain, up to the
    // counter block's capacity (paths still alive after that many vertices are cut).
    uint32_t const bounce_iterations = settings_.max_bounces + 1;
    uint32_t const max_iterations = d_->has_media ? Max_bounce_slots - 1 : bounce_iterations;

    stats_                  = Stats();
    stats_.instances        = instances_;
    stats_.device_triangles = device_triangles_;
    if (settings_.spectral) {
        return render_spectral(&sg, first_sample, num_samples);
    }
    std::vector<uint32_t> host_ctr(Counter_words);
    // Device time of the guide's stages: event pairs (inference after each trace, training
    // after each pass), summed after each wave.
    auto const guide_event = [&](size_t i) {
        while (d_->guide_events.size() <= i) {
            cudaEvent_t e = nullptr;
            cudaEventCreate(&e);
            d_->guide_events.push_back(e);
        }
        return d_->guide_events[i];
    };
    if (!d_->launch_dev) {
        SPB_RCUDA(dev_malloc(&d_->launch_dev, sizeof(Launch)));
        SPB_RCUDA(cudaMallocHost(&d_->launch_host, sizeof(Launch)));
    }
    auto const record = [&](cudaEvent_t e, bool capture) {
        return capture ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal) : cudaEventRecord(e, st);
    };
    bool const guide_at_all = settings_.guiding;
    auto const guided_at    = [&](uint32_t b) { return guide_at_all && (d_->has_media || b < settings_.guide_depth); };

    // Enqueues one wave's kernels (its launch block already copied to the device): generate,
    // then per vertex extend / guide / shade / shadow, the guide's training after a training
    // pass, and the film gather.  With media the bounce loop checks the extension queue on the
    // host, so such waves are never captured into a graph.
    auto const enqueue_wave = [&](uint32_t k, uint32_t paths, uint32_t trace_grid, bool training, bool capture,
                                  uint32_t& iterations, size_t& events) -> int32_t {
        SPB_RCUDA(cudaMemsetAsync(ctr, 0, Counter_words * sizeof(uint32_t), st));
        // k_transmit: one thread per shadow slot (at most two per path)
        uint32_t const transmit_grid = (2 * paths + Trace_block - 1) / Trace_block;
        k_generate<<<(paths + 255) / 256, 256, 0, st>>>(d_->launch_dev, d_->paths, d_->queue[0], ctr, paths);
        iterations = 0;
        for (uint32_t b = 0; b < max_iterations; ++b) {
            if (b >= bounce_iterations) {
                SPB_RCUDA(cudaMemcpyAsync(d_->pinned_count, ctr + Counter_stride * b, sizeof(uint32_t),
                                          cudaMemcpyDeviceToHost, st));
                SPB_RCUDA(cudaStreamSynchronize(st));
                if (*d_->pinned_count == 0) {
                    break;
                }
            }
            iterations               = b + 1;
            uint32_t* const q_in  = d_->queue[b & 1];
            uint32_t* const q_out = d_->queue[(b + 1) & 1];
            uint32_t* const c     = ctr + Counter_stride * b;
            if (d_->instanced) {
                k_trace<false, false, true><<<trace_grid, Trace_block, 0, st>>>(sg, d_->paths, q_in, c, c + 2,
                                                                               ctr + Overflow_slot);
            } else {
                k_trace<false><<<trace_grid, Trace_block, 0, st>>>(sg, d_->paths, q_in, c, c + 2, ctr + Overflow_slot);
            }
            // (without media a vertex's depth is the iteration; with media it can be less)
            if (guided_at(b)) {
                SPB_RCUDA(record(guide_event(events++), capture));
                k_guide_encode<<<(paths + 255) / 256, 256, 0, st>>>(sg, d_->launch_dev, d_->paths, q_in, c);
                k_guide<<<d_->guide_grid, guide::Block, sizeof(Infer_smem), st>>>(
                    d_->paths, c, d_->net.weights(), d_->net.parameters(), ctr + Overflow_slot + 1);
                SPB_RCUDA(record(guide_event(events++), capture));
            }
            k_shade<<<(paths + Shade_block - 1) / Shade_block, Shade_block, 0, st>>>(
                sg, d_->launch_dev, d_->paths, q_in, c,
                Shade_out{q_out, c + Counter_stride, d_->shadow_queue, c + 1, c + 5, c + 6});
            if (d_->has_media) {
                Transmit_out const tq{d_->transmit_queue, c + 4, c + 8, 2 * paths, d_->transmit_pick_queue, c + 7};
                if (d_->instanced) {
                    k_trace<true, true, true><<<trace_grid, Trace_block, 0, st>>>(
                        sg, d_->paths, d_->shadow_queue, c + 1, c + 3, ctr + Overflow_slot, tq);
                    k_transmit<true><<<transmit_grid, Trace_block, 0, st>>>(sg, d_->paths, d_->transmit_queue, c + 4,
                                                                            c + 8, 2 * paths, ctr + Overflow_slot);
                } else {
                    k_trace<true, true><<<trace_grid, Trace_block, 0, st>>>(sg, d_->paths, d_->shadow_queue, c + 1,
                                                                           c + 3, ctr + Overflow_slot, tq);
                    k_transmit<false><<<transmit_grid, Trace_block, 0, st>>>(sg, d_->paths, d_->transmit_queue, c + 4,
                                                                             c + 8, 2 * paths, ctr + Overflow_slot);
                }
                if (picks_per_path != 0) {
                    // picks through media, one thread each: their number sets the grid (waves
                    // with media read counters on the host and are never captured)
                    SPB_RCUDA(cudaMemcpyAsync(d_->pinned_count, c + 7, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
                    SPB_RCUDA(cudaStreamSynchronize(st));
                    uint32_t const picked = *d_->pinned_count;
                    if (picked != 0 && d_->instanced) {
                        k_transmit_picks<true><<<(picked + Trace_block - 1) / Trace_block, Trace_block, 0, st>>>(
                            sg, d_->paths, d_->transmit_pick_queue, c + 7, ctr + Overflow_slot);
                    } else if (picked != 0) {
                        k_transmit_picks<false><<<(picked + Trace_block - 1) / Trace_block, Trace_block, 0, st>>>(
                            sg, d_->paths, d_->transmit_pick_queue, c + 7, ctr + Overflow_slot);
                    }
                }
            } else if (d_->instanced) {
                k_trace<true, false, true><<<trace_grid, Trace_block, 0, st>>>(sg, d_->paths, d_->shadow_queue, c + 1,
                                                                              c + 3, ctr + Overflow_slot);
            } else {
                k_trace<true><<<trace_grid, Trace_block, 0, st>>>(sg, d_->paths, d_->shadow_queue, c + 1, c + 3,
                                                                  ctr + Overflow_slot);
            }
            if (picks_per_path != 0) {
                k_pick_sum<<<std::min((paths + 255) / 256, 8 * d_->sms), 256, 0, st>>>(d_->paths, c + 6);
            }
        }
        if (training) {
            SPB_RCUDA(record(guide_event(events++), capture));
            if (int32_t const e = train_guide(paths)) {
                return e;
            }
            SPB_RCUDA(record(guide_event(events++), capture));
        }
        k_gather<<<(d_->film_pixels + 255) / 256, 256, 0, st>>>(d_->paths, d_->launch_dev, d_->film_pixels, k,
                                                                d_->film, d_->comp);
        SPB_RCUDA(cudaGetLastError());
        return SPB_OK;
    };

    if (settings_.guiding) {
        guide_event(2 * Max_bounce_slots + 2);  // every event a wave can use, created before any capture
    }
    SPB_RCUDA(cudaEventRecord(d_->ev0, st));
    for (uint32_t done = 0; done < num_samples;) {
        bool const training = settings_.guiding &&
                              (settings_.guide_train_spp == 0 || first_sample + done < settings_.guide_train_spp);
        // this wave's configuration: tuned, the tuner's current candidate, or the settings
        Tuner const&   tn          = d_->tuner;
        bool const     probe       = tuning && !training && !tn.done();
        uint32_t const wave_paths  = std::min(settings_.wave_paths ? settings_.wave_paths
                                                                   : (tn.done() ? tn.best_wave : tn.wave_paths),
                                              max_paths);
        uint32_t const blocks_sm   = settings_.trace_blocks_per_sm
                                         ? std::min(settings_.trace_blocks_per_sm, tn.max_per_sm)
                                         : (tn.done() ? tn.best_sm : (training ? tn.max_per_sm : tn.per_sm));
        uint32_t const trace_grid  = blocks_sm * d_->sms;
        uint32_t const full_k      = training ? train_wave : wave_spp(wave_paths);
        uint32_t const k           = std::min(full_k, num_samples - done);
        bool const     measured    = probe && k == full_k;  // a full wave of the candidate
        uint32_t const paths       = k * pixels;
        Wave           wave{first_sample + done, k, settings_.seed, settings_.min_bounces,
                  settings_.max_bounces};
        wave.guiding        = settings_.guiding ? 1u : 0u;
        wave.guide_fraction = settings_.guide_fraction;
        wave.metal_fraction = settings_.metal_fraction < 0.f ? settings_.guide_fraction : settings_.metal_fraction;
        wave.guide_depth    = settings_.guide_depth;
        wave.record_depth   = training ? settings_.record_depth : 0u;
        wave.bounds_lo      = d_->bounds_lo;
        wave.bounds_inv     = d_->bounds_inv;
        wave.golden_n       = golden_n;
        wave.golden_sorted  = d_->golden_sorted;
        // The previous wave has completed (synchronized below), so the pinned block is free.
        d_->launch_host->cams         = d_->cams;
        d_->launch_host->view_offsets = d_->view_offsets;
        d_->launch_host->film_offsets = d_->film_offsets;
        d_->launch_host->num_views    = d_->num_views;
        d_->launch_host->pixels       = pixels;
        d_->launch_host->wave         = wave;
        if (measured) {
            SPB_RCUDA(cudaEventRecord(d_->wave_ev[0], st));
        }
        SPB_RCUDA(cudaMemcpyAsync(d_->launch_dev, d_->launch_host, sizeof(Launch), cudaMemcpyHostToDevice, st));
        uint32_t iterations = 0;
        size_t   events     = 0;
        // Wave shapes that recur are replayed from graphs: a shape is captured when it comes the
        // second time (waves without media or training, up to Graph_max_paths paths).
        Device::Wave_graph* g = nullptr;
        bool const graphable = settings_.cuda_graphs && !d_->has_media && !training && paths <= Graph_max_paths;
        if (graphable) {
            for (auto& e : d_->graphs) {
                if (e.k == k && e.trace_grid == trace_grid) {
                    g = &e;
                }
            }
            if (!g) {
                d_->graphs.push_back({k, trace_grid, 0, 0, nullptr});  // first sighting
            }
        }
        if (g) {
            if (!g->exec) {
                SPB_RCUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                int32_t const     e     = enqueue_wave(k, paths, trace_grid, false, true, iterations, events);
                cudaGraph_t       graph = nullptr;
                cudaError_t const ce    = cudaStreamEndCapture(st, &graph);
                if (e != SPB_OK || ce != cudaSuccess) {
                    if (graph) {
                        cudaGraphDestroy(graph);
                    }
                    return e != SPB_OK ? e : fail_cuda("cudaStreamEndCapture", int(ce));
                }
                cudaGraphExec_t   exec = nullptr;
                cudaError_t const ie   = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                SPB_RCUDA(ie);
                *g = Device::Wave_graph{k, trace_grid, iterations, uint32_t(events), exec};
            }
            SPB_RCUDA(cudaGraphLaunch(g->exec, st));
            iterations = g->iterations;
            events     = g->events;
            ++stats_.graph_waves;
        } else if (int32_t const e = enqueue_wave(k, paths, trace_grid, training, false, iterations, events)) {
            return e;
        }
        if (measured) {
            SPB_RCUDA(cudaEventRecord(d_->wave_ev[1], st));
        }
        SPB_RCUDA(cudaMemcpyAsync(host_ctr.data(), ctr, Counter_words * sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, st));
        SPB_RCUDA(cudaStreamSynchronize(st));
        if (measured) {
            float wave_ms = 0.f;
            SPB_RCUDA(cudaEventElapsedTime(&wave_ms, d_->wave_ev[0], d_->wave_ev[1]));
            d_->tuner.report(double(wave_ms) * 1e6 / double(paths));
        }
        // the guide's stages of this wave: inference pairs, then the training pair
        for (size_t i = 0; i + 1 < events; i += 2) {
            float pair_ms = 0.f;
            cudaEventElapsedTime(&pair_ms, d_->guide_events[i], d_->guide_events[i + 1]);
            bool const train = training && i + 2 == events;
            (train ? stats_.guide_training_seconds : stats_.guide_inference_seconds) += double(pair_ms) * 1e-3;
        }
        if (training) {
            stats_.guide_training_samples += uint64_t(settings_.guide_steps) * settings_.guide_batch;
        }
        for (uint32_t b = 0; b < iterations; ++b) {
            stats_.extension_rays += host_ctr[Counter_stride * b];
            stats_.shadow_rays += host_ctr[Counter_stride * b + 1];
            if (guided_at(b)) {
                stats_.guide_vertices += host_ctr[Counter_stride * b];
            }
        }
        stats_.overflow += host_ctr[Overflow_slot];
        stats_.tracking_capped += host_ctr[Overflow_slot + 2];
        if (host_ctr[Overflow_slot + 1]) {
            error_ = "path guiding: a tensor-core completion wait ran out";
            return SPB_ERROR_CUDA;
        }
        stats_.paths += paths;
        stats_.wave_paths          = std::max(stats_.wave_paths, paths);
        stats_.trace_blocks_per_sm = blocks_sm;
        done += k;
    }
    SPB_RCUDA(cudaEventRecord(d_->ev1, st));
    SPB_RCUDA(cudaEventSynchronize(d_->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, d_->ev0, d_->ev1);
    stats_.seconds = double(ms) * 1e-3;
    return SPB_OK;
}

// Spectral mode: one persistent launch over every (view, pixel, sample) of the call, its
// samples splatted into the views' films (see k_spectral).
int32_t Renderer::render_spectral(void const* scene, uint32_t first_sample, uint32_t num_samples) {
    Scene_gpu const&   sg = *static_cast<Scene_gpu const*>(scene);
    cudaStream_t const st = d_->stream;
    if (!d_->spectral_table) {
        double c[9];
        double m[9];
        for (int i = 0; i < 9; ++i) {
            m[i] = spectral::Srgb_to_ap1[i];
        }
        spectral::readout_matrix(m, c);
        std::vector<float> table(3 * Spec_table);
        for (int i = 0; i < Spec_table; ++i) {
            double resp[3];
            spectral::response(spectral::Lambda_min + double(i), m, resp);
            for (int k = 0; k < 3; ++k) {
                table[3 * i + k] = float((c[3 * k] * resp[0] + c[3 * k + 1] * resp[1] + c[3 * k + 2] * resp[2]) *
                                         double(spectral::Lambda_span) / spectral::Hero_count);
            }
        }
        SPB_RCUDA(cudaMemcpyToSymbol(c_spec_resp, table.data(), table.size() * sizeof(float)));
        d_->spectral_table = true;
    }
    if (!d_->spectral_work) {
        SPB_RCUDA(dev_malloc(&d_->spectral_work, 4 * sizeof(unsigned long long)));
    }
    if (!d_->launch_dev) {
        SPB_RCUDA(dev_malloc(&d_->launch_dev, sizeof(Launch)));
        SPB_RCUDA(cudaMallocHost(&d_->launch_host, sizeof(Launch)));
    }
    // With guiding, the first guide_train_spp samples (at most half of the call's) train the
    // phase guide, a fit turns its sums into lobes, and the rest are guided by them.
    uint32_t const cells = uint32_t(Phase_cells) * Phase_cells * Phase_cells;
    uint32_t const train = settings_.guiding ? std::min(std::max(settings_.guide_train_spp, 1u), num_samples / 2) : 0u;
    Phase_guide    pg{};
    if (train != 0) {
        if (!d_->phase_sums) {
            SPB_RCUDA(dev_malloc(&d_->phase_sums, cells * sizeof(float4)));
            SPB_RCUDA(dev_malloc(&d_->phase_counts, cells * sizeof(uint32_t)));
            SPB_RCUDA(dev_malloc(&d_->phase_lobes, cells * sizeof(float4)));
        }
        SPB_RCUDA(cudaMemsetAsync(d_->phase_sums, 0, cells * sizeof(float4), st));
        SPB_RCUDA(cudaMemsetAsync(d_->phase_counts, 0, cells * sizeof(uint32_t), st));
        pg.sums     = d_->phase_sums;
        pg.counts   = d_->phase_counts;
        pg.lobes    = d_->phase_lobes;
        pg.lo       = d_->bounds_lo;
        pg.scale    = make_float4(d_->bounds_inv.x * Phase_cells, d_->bounds_inv.y * Phase_cells,
                                  d_->bounds_inv.z * Phase_cells, 0.f);
        pg.n        = Phase_cells;
        pg.fraction = settings_.guide_fraction;
    }
    SPB_RCUDA(cudaMemsetAsync(d_->spectral_work, 0, 4 * sizeof(unsigned long long), st));
    SPB_RCUDA(cudaMemsetAsync(d_->counters, 0, Counter_words * sizeof(uint32_t), st));
    d_->launch_host->cams         = d_->cams;
    d_->launch_host->view_offsets = d_->view_offsets;
    d_->launch_host->film_offsets = d_->film_offsets;
    d_->launch_host->num_views    = d_->num_views;
    d_->launch_host->pixels       = d_->traced_pixels;
    // One persistent launch over samples [first, first + count) of every pixel of every view.
    auto const launch = [&](int mode, uint32_t first, uint32_t count) -> int32_t {
        // the launch block's pinned copy is free once the previous launch's copy has run
        SPB_RCUDA(cudaStreamSynchronize(st));
        d_->launch_host->wave = Wave{first, count, settings_.seed, settings_.min_bounces, settings_.max_bounces};
        SPB_RCUDA(cudaMemcpyAsync(d_->launch_dev, d_->launch_host, sizeof(Launch), cudaMemcpyHostToDevice, st));
        SPB_RCUDA(cudaMemsetAsync(d_->spectral_work, 0, sizeof(unsigned long long), st));
        uint64_t const n      = uint64_t(d_->traced_pixels) * count;
        int            per_sm = 0;
        auto const     kernel = mode == Spectral_train ? k_spectral<Spectral_train>
                                : mode == Spectral_guided ? k_spectral<Spectral_guided>
                                                          : k_spectral<Spectral_plain>;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, Trace_block, 0);
        uint32_t const grid = uint32_t(std::max(1, per_sm)) * d_->sms;
        kernel<<<grid, Trace_block, 0, st>>>(sg, d_->launch_dev, n, d_->spectral_work, d_->film,
                                             d_->counters + Overflow_slot, d_->spectral_work + 2, pg);
        SPB_RCUDA(cudaGetLastError());
        return SPB_OK;
    };
    uint64_t const total = uint64_t(d_->traced_pixels) * num_samples;
    SPB_RCUDA(cudaEventRecord(d_->ev0, st));
    if (train == 0) {
        if (int32_t const e = launch(Spectral_plain, first_sample, num_samples)) {
            return e;
        }
    } else {
        if (int32_t const e = launch(Spectral_train, first_sample, train)) {
            return e;
        }
        k_phase_fit<<<(cells + 255) / 256, 256, 0, st>>>(pg, d_->phase_lobes);
        SPB_RCUDA(cudaGetLastError());
        if (int32_t const e = launch(Spectral_guided, first_sample + train, num_samples - train)) {
            return e;
        }
    }
    SPB_RCUDA(cudaEventRecord(d_->ev1, st));
    unsigned long long counts[4];
    uint32_t           host_ctr[4];
    SPB_RCUDA(cudaMemcpyAsync(counts, d_->spectral_work, sizeof(counts), cudaMemcpyDeviceToHost, st));
    SPB_RCUDA(cudaMemcpyAsync(host_ctr, d_->counters + Overflow_slot, sizeof(host_ctr), cudaMemcpyDeviceToHost, st));
    SPB_RCUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, d_->ev0, d_->ev1);
    stats_.seconds         = double(ms) * 1e-3;
    stats_.paths           = total;
    stats_.extension_rays  = counts[2];
    stats_.shadow_rays     = counts[3];
    stats_.overflow        = host_ctr[0];
    stats_.tracking_capped = host_ctr[2];
    stats_.wave_paths      = uint32_t(std::min<uint64_t>(total, 0xFFFFFFFFu));
    return SPB_OK;
}

int32_t Renderer::resolve(float* rgba) {
    if (!d_->film) {
        error_ = "no camera";
        return SPB_ERROR_STATE;
    }
    uint32_t const n = d_->film_pixels;
    k_resolve<<<(n + 255) / 256, 256, 0, d_->stream>>>(d_->film, d_->comp, n, d_->out);
    SPB_RCUDA(cudaGetLastError());
    SPB_RCUDA(cudaMemcpyAsync(rgba, d_->out, n * sizeof(float4), cudaMemcpyDeviceToHost,
                              d_->stream));
    SPB_RCUDA(cudaStreamSynchronize(d_->stream));
    return SPB_OK;
}

}  // namespace spb::render
