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

#include "bvh8.hpp"
#include "common.hpp"
#include "ggx_table.hpp"
#include "render.hpp"
#include "traverse.cuh"

namespace spb::render {

namespace {

using shading::V3;
using shading::v3;

constexpr uint32_t Full_mask        = 0xFFFFFFFFu;
constexpr int      Trace_block      = 128;
constexpr int      Shade_block      = 256;
constexpr uint32_t Refill_threshold = 8;
constexpr float    Ray_max_t        = 3.4027715434167032e+38f;
constexpr int      Filter_samples   = 30;
constexpr uint32_t Max_bounce_slots = 64;
constexpr uint32_t Class_surface    = 1;  // Wide_triangle::tri_class of ordinary surfaces
constexpr uint32_t Class_boundary   = 2;  // ... of participating-medium boundaries

// Counter block (uint32): per bounce b, [8b] extension count, [8b+1] shadow count,
// [8b+2] extend fetch, [8b+3] shadow fetch, [8b+4] transmittance count; then the overflow
// counter.
constexpr uint32_t Counter_stride = 8;
constexpr uint32_t Counter_words  = Counter_stride * Max_bounce_slots + 4;
constexpr uint32_t Overflow_slot  = Counter_stride * Max_bounce_slots;

struct Scene_gpu {
    uint4 const*              nodes;
    float4 const*             tris;
    float                     hit_margin;
    uint4 const*              tri_info;  // v0, v1, v2, material
    float4 const*             positions;
    float4 const*             normals;
    shading::Material const*  materials;
    float const*              tri_light_pdf;  // pick probability / area, 0 if not a sampled light
    float4 const*             lights;         // 3 per light: (a, area), (e1, pick), (e2, tri id)
    float const*              light_cdf;      // num_lights + 1 entries
    uint32_t                  num_lights;
    float const*              e_table;
};

struct Paths {
    float4*   ray_o;  // origin, min_t
    float4*   ray_d;  // direction, max_t
    uint32_t* hit_id;
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
};

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
};

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

__device__ __forceinline__ V3 f3v(float4 a) {
    return v3(a.x, a.y, a.z);
}

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

// ---- generate: camera rays (Perspective::generate_ray, camera_perspective.cpp:47-80) ----
__global__ void k_generate(Cam cam, Wave wave, Paths p, uint32_t* queue, uint32_t* counters,
                           uint32_t num_paths) {
    uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        counters[0] = num_paths;
    }
    if (i >= num_paths) {
        return;
    }
    uint32_t const pixels = cam.w * cam.h;
    uint32_t const pixel  = i % pixels;
    uint32_t const slot   = i / pixels;
    uint32_t const x      = pixel % cam.w;
    uint32_t const y      = pixel / cam.w;

    Rng rng;
    rng.start(wave.seed, uint64_t(pixel) + uint64_t(wave.first_sample + slot) * pixels);
    float const u = rng.uniform();
    float const v = rng.uniform();

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
    p.puv[i]   = make_float2(u, v);
    p.rng[i]   = rng.save();
    p.info[i]  = 1u << 16;  // vertex 0, depth 0, treat as singular
    queue[i]   = i;
}

// ---- extend / shadow: persistent traversal over a queue of path indices ----
// Any_hit: shadow rays.  Media: the scene has participating media -- shadow rays ignore
// medium boundaries and unoccluded ones go to the transmittance queue instead of adding
// their contribution directly.
template <bool Any_hit, bool Media = false>
__global__ void __launch_bounds__(Trace_block)
    k_trace(Scene_gpu s, Paths p, uint32_t const* __restrict__ queue,
            uint32_t const* __restrict__ count, uint32_t* fetch, uint32_t* overflow,
            uint32_t* transmit_queue = nullptr, uint32_t* transmit_count = nullptr) {
    uint32_t const num  = *count;
    uint32_t const lane = threadIdx.x & 31u;
    uint32_t const lt   = (1u << lane) - 1u;

    gpu::Ray_state r;
    gpu::Traversal tv;
    uint2          stack[gpu::Stack_size];
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
                        gpu::start_ray(r, tv, p.sh_o[path], p.sh_d[path]);
                    } else {
                        gpu::start_ray(r, tv, p.ray_o[path], p.ray_d[path]);
                    }
                    active = true;
                }
            }
        }
        if (!active) {
            continue;
        }
        if (gpu::traversal_step<Any_hit, Media>(r, tv, stack, s.nodes, s.tris, s.hit_margin,
                                                 overflow, Class_boundary)) {
            if (Any_hit) {
                if (r.best_id == gpu::Miss) {
                    if (Media) {
                        transmit_queue[atomicAdd(transmit_count, 1u)] = path;
                    } else {
                        float4 const c = p.sh_L[path];
                        float4       l = p.L[path];
                        l.x += c.x;
                        l.y += c.y;
                        l.z += c.z;
                        p.L[path] = l;
                    }
                }
            } else {
                p.hit_id[path] = r.best_id;
                p.hit_t[path]  = r.tbest;
                p.hit_uv[path] = make_float2(r.u, r.v);
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

// Light sample for next-event estimation seen from ps: power-proportional triangle, uniform
// point, solid-angle pdf (with the pick probability).  False if the sample is unusable
// (grazing or behind a one-sided emitter, Mesh::sample in triangle_mesh.cpp:462-516).
struct Light_sample {
    V3    dir;
    float dist;
    float pdf;
    V3    radiance;
};

__device__ __forceinline__ bool sample_light(Scene_gpu const& s, V3 ps, float r, float r1, float r2,
                                             Light_sample& ls) {
    uint32_t lo = 0;
    uint32_t hi = s.num_lights;
    while (hi - lo > 1) {
        uint32_t const mid = (lo + hi) >> 1;
        if (s.light_cdf[mid] <= r) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    float4 const   la   = s.lights[3 * lo + 0];
    float4 const   le1  = s.lights[3 * lo + 1];
    float4 const   le2  = s.lights[3 * lo + 2];
    uint32_t const ltri = __float_as_uint(le2.w);
    float const    sq   = sqrtf(r1);
    V3 const       q    = f3v(la) + (sq * (1.f - r2)) * f3v(le1) + (sq * r2) * f3v(le2);
    V3             ln   = shading::normalize(shading::cross(f3v(le1), f3v(le2)));
    shading::Material const lmat = s.materials[s.tri_info[ltri].w];
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
    ls.pdf      = le1.w * d2 / (cl * la.w);
    ls.radiance = lmat.emission;
    return true;
}

// Homogeneous-medium tracking over [t, d] with spectral MIS (Tracking::tracking for a
// homogeneous medium, tracking.cpp:425-470): returns true on a scattering event at t_out;
// lw receives the path weight either way.
__device__ __forceinline__ bool track_homogeneous(shading::Material const& m, float t, float d,
                                                  Rng& rng, float& t_out, V3& lw) {
    V3 const    mu_t = m.mu_a + m.mu_s;
    float const mt   = shading::max_component(mu_t);
    lw               = v3(1.f, 1.f, 1.f);
    if (!(mt > 1e-10f)) {
        return false;
    }
    float const imt  = 1.f / mt;
    V3 const    mu_n = v3(mt - mu_t.x, mt - mu_t.y, mt - mu_t.z);
    for (int step = 0; step < 4096; ++step) {
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
    return false;
}

// ---- shade: one path vertex ----
__global__ void __launch_bounds__(Shade_block)
    k_shade(Scene_gpu s, Wave wave, Paths p, uint32_t const* __restrict__ q_in,
            uint32_t const* __restrict__ count_in, uint32_t* q_out, uint32_t* count_out,
            uint32_t* sq, uint32_t* count_shadow) {
    uint32_t const i   = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t const num = *count_in;

    bool     extend = false;
    bool     shadow = false;
    uint32_t path   = 0;

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
            done = true;
        } else if (medium != 0) {
            shading::Material const m = s.materials[medium - 1];
            V3 lw;
            scatter = track_homogeneous(m, ro.w, p.hit_t[path], rng, t_sc, lw);
            T       = T * lw;
            if (!(lw.x >= Abort_epsilon || lw.y >= Abort_epsilon || lw.z >= Abort_epsilon)) {
                done = true;
            }
        }

        if (!done && scatter) {
            // Scattering vertex inside the medium (volumetric::Sample, HG phase function).
            if (depth >= wave.max_bounces) {
                done = true;
            } else if (depth >= wave.min_bounces) {
                float const q = shading::max_component(T);
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
                if (s.num_lights > 0) {
                    float const  r  = rng.uniform();
                    float const  r1 = rng.uniform();
                    float const  r2 = rng.uniform();
                    Light_sample ls;
                    if (sample_light(s, pos, r, r1, r2, ls)) {
                        float const f = shading::phase_hg(shading::dot(wo, ls.dir), g);
                        float const w = ls.pdf / (ls.pdf * ls.pdf + f * f);
                        V3 const contrib = (w * f) * (T * ls.radiance);
                        if (shading::max_component(contrib) > 0.f) {
                            p.sh_o[path] = make_float4(pos.x, pos.y, pos.z, 0.f);
                            p.sh_d[path] = make_float4(ls.dir.x, ls.dir.y, ls.dir.z, ls.dist);
                            p.sh_L[path] = make_float4(contrib.x, contrib.y, contrib.z, 0.f);
                            shadow       = true;
                        }
                    }
                }
                float const x0 = rng.uniform();
                float const x1 = rng.uniform();
                float       pdf;
                V3 const    wi = shading::sample_hg(wo, g, x0, x1, pdf);
                p.ray_o[path]  = make_float4(pos.x, pos.y, pos.z, 0.f);
                p.ray_d[path]  = make_float4(wi.x, wi.y, wi.z, Ray_max_t);
                bsdf_pdf       = pdf;  // reflection / pdf == 1
                singular       = false;
                ++depth;
                ++vtx;
                extend = true;
            }
        } else if (!done) {
            uint4 const  tri = s.tri_info[id];
            V3 const     a   = f3v(s.positions[tri.x]);
            V3 const     b   = f3v(s.positions[tri.y]);
            V3 const     c   = f3v(s.positions[tri.z]);
            float2 const uv  = p.hit_uv[path];
            float const  bw  = 1.f - uv.x - uv.y;
            V3 const     pos = bw * a + uv.x * b + uv.y * c;
            V3           geo_n = shading::normalize(shading::cross(b - a, c - a));
            V3 const     na  = f3v(s.normals[tri.x]);
            V3 const     nb  = f3v(s.normals[tri.y]);
            V3 const     nc  = f3v(s.normals[tri.z]);
            V3           ns  = shading::normalize(bw * na + uv.x * nb + uv.y * nc);
            V3 const     wo  = -dir_in;
            shading::Material const mat = s.materials[tri.w];
            float const  cos_o = shading::dot(geo_n, wo);
            bool const   front = cos_o > 0.f;
            bool const   emits = mat.type == shading::Type_light;

            if (vtx > 0) {
                // Emission reached by the BSDF sample (connect_light, pathtracer_mis.cpp:349-380).
                if (emits) {
                    if (front || mat.two_sided) {
                        float w = 1.f;
                        if (!singular) {
                            float const t      = p.hit_t[path];
                            float const pdf_l  = s.tri_light_pdf[id] * (t * t) / fabsf(cos_o);
                            w                  = power_heuristic(bsdf_pdf, pdf_l);
                        }
                        L = L + w * (T * mat.emission);
                    }
                    done = true;
                } else if (depth >= wave.max_bounces) {
                    done = true;
                } else if (depth >= wave.min_bounces) {
                    float const q = shading::max_component(T);
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
                medium        = front ? tri.w + 1 : 0;
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

                // Next-event estimation (sample_lights / evaluate_light, pathtracer_mis.cpp:281-347).
                if (s.num_lights > 0) {
                    float const  r  = rng.uniform();
                    float const  r1 = rng.uniform();
                    float const  r2 = rng.uniform();
                    V3 const     ps = offset_ray(pos, geo_n);
                    Light_sample ls;
                    if (sample_light(s, ps, r, r1, r2, ls)) {
                        shading::Bxdf const f =
                            shading::substitute_evaluate(mat, s.e_table, ctx, ls.dir);
                        float const w = ls.pdf / (ls.pdf * ls.pdf + f.pdf * f.pdf);
                        V3 const contrib = w * (T * (ls.radiance * f.reflection));
                        if (shading::max_component(contrib) > 0.f) {
                            p.sh_o[path] = make_float4(ps.x, ps.y, ps.z, 0.f);
                            p.sh_d[path] = make_float4(ls.dir.x, ls.dir.y, ls.dir.z, ls.dist);
                            p.sh_L[path] = make_float4(contrib.x, contrib.y, contrib.z, 0.f);
                            shadow       = true;
                        }
                    }
                }

                // BSDF sample (pathtracer_mis.cpp:153-201).
                float const xl = rng.uniform();
                float const x0 = rng.uniform();
                float const x1 = rng.uniform();
                shading::Sampled const smp =
                    shading::substitute_sample(mat, s.e_table, ctx, xl, x0, x1);
                if (smp.pdf > 0.f) {
                    V3 const o = offset_ray(pos, shading::dot(geo_n, smp.wi) > 0.f ? geo_n : -geo_n);
                    p.ray_o[path] = make_float4(o.x, o.y, o.z, 0.f);
                    p.ray_d[path] = make_float4(smp.wi.x, smp.wi.y, smp.wi.z, Ray_max_t);
                    T        = (1.f / smp.pdf) * (T * smp.reflection);
                    bsdf_pdf = smp.pdf;
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

    uint32_t const slot = append(count_out, extend);
    if (extend) {
        q_out[slot] = path;
    }
    uint32_t const sslot = append(count_shadow, shadow);
    if (shadow) {
        sq[sslot] = path;
    }
}

// ---- shadow rays through media: Worker::transmittance (rendering_worker.cpp:209-267) ----
// For each unoccluded shadow ray of a scene with media, walks the medium boundaries along the
// ray (closest hits on boundary triangles only), accumulates the optical depth of each
// homogeneous segment, and adds exp(-optical depth) times the light contribution.
__global__ void __launch_bounds__(Trace_block)
    k_transmit(Scene_gpu s, Paths p, uint32_t const* __restrict__ queue,
               uint32_t const* __restrict__ count, uint32_t* overflow) {
    uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count) {
        return;
    }
    uint32_t const path   = queue[i];
    uint32_t       medium = p.info[path] >> 17;
    float4 const   ro     = p.sh_o[path];
    float4 const   rd     = p.sh_d[path];
    float          t0     = ro.w;
    V3             tau    = v3(0.f, 0.f, 0.f);
    uint2          stack[gpu::Stack_size];
    for (int crossing = 0; crossing < 64; ++crossing) {
        gpu::Ray_state r;
        gpu::Traversal tv;
        gpu::start_ray(r, tv, make_float4(ro.x, ro.y, ro.z, t0), rd);
        while (!gpu::traversal_step<false, true>(r, tv, stack, s.nodes, s.tris, s.hit_margin,
                                                 overflow, Class_surface)) {
        }
        bool const  hit = r.best_id != gpu::Miss;
        float const end = hit ? r.tbest : rd.w;
        if (medium != 0) {
            shading::Material const m = s.materials[medium - 1];
            float const len = fmaxf(end - t0, 0.f);
            tau = tau + len * (m.mu_a + m.mu_s);
        }
        if (!hit) {
            break;
        }
        uint4 const tri = s.tri_info[r.best_id];
        V3 const    a   = f3v(s.positions[tri.x]);
        V3 const    geo = shading::cross(f3v(s.positions[tri.y]) - a, f3v(s.positions[tri.z]) - a);
        medium          = shading::dot(geo, v3(rd.x, rd.y, rd.z)) < 0.f ? tri.w + 1 : 0;
        t0              = offset_f(r.tbest);
        if (t0 >= rd.w) {
            break;
        }
    }
    float4 const c = p.sh_L[path];
    float4       l = p.L[path];
    l.x += expf(-tau.x) * c.x;
    l.y += expf(-tau.y) * c.y;
    l.z += expf(-tau.z) * c.z;
    p.L[path] = l;
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

__global__ void k_gather(Paths p, uint32_t w, uint32_t h, uint32_t samples, float4* film,
                         float4* comp) {
    uint32_t const q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= w * h) {
        return;
    }
    int const x = int(q % w);
    int const y = int(q / w);
    float4    acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int dy = -1; dy <= 1; ++dy) {
        int const sy = y - dy;
        if (sy < 0 || sy >= int(h)) {
            continue;
        }
        for (int dx = -1; dx <= 1; ++dx) {
            int const sx = x - dx;
            if (sx < 0 || sx >= int(w)) {
                continue;
            }
            uint32_t const src = uint32_t(sy) * w + uint32_t(sx);
            for (uint32_t k = 0; k < samples; ++k) {
                uint32_t const path = k * w * h + src;
                float2 const   uv   = p.puv[path];
                float const    wt   = filter_weight(uv.x - 0.5f - float(dx)) *
                                 filter_weight(uv.y - 0.5f - float(dy));
                float4 const L = p.L[path];
                acc.x += wt * L.x;
                acc.y += wt * L.y;
                acc.z += wt * L.z;
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
    float*             tri_light_pdf = nullptr;
    float4*            lights     = nullptr;
    float*             light_cdf  = nullptr;
    float*             e_table    = nullptr;
    uint32_t           num_lights = 0;
    float              hit_margin = 0.f;
    // paths
    uint32_t  capacity = 0;
    Paths     paths{};
    uint32_t* queue[2] = {nullptr, nullptr};
    uint32_t* shadow_queue   = nullptr;
    uint32_t* transmit_queue = nullptr;
    uint32_t* counters       = nullptr;
    bool      has_media      = false;
    // film
    float4*   film = nullptr;
    float4*   comp = nullptr;
    float4*   out  = nullptr;
    uint32_t  film_pixels = 0;
    int       trace_grid  = 0;
    cudaStream_t stream   = nullptr;
    cudaEvent_t  ev0      = nullptr;
    cudaEvent_t  ev1      = nullptr;
};

namespace {

template <typename T>
void free_ptr(T*& p) {
    if (p) {
        cudaFree(p);
        p = nullptr;
    }
}

template <typename T>
cudaError_t upload(T*& dst, void const* src, size_t bytes) {
    free_ptr(dst);
    cudaError_t e = cudaMalloc(&dst, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) {
        return e;
    }
    return bytes ? cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
}

}  // namespace

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
    cudaEventCreate(&d_->ev0);
    cudaEventCreate(&d_->ev1);
    int per_sm = 0;
    int sms    = 0;
    int dev    = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace<false>, Trace_block, 0);
    d_->trace_grid = std::max(1, per_sm) * std::max(1, sms);
}

Renderer::~Renderer() {
    if (!d_) {
        return;
    }
    cudaDeviceSynchronize();
    free_ptr(d_->nodes);
    free_ptr(d_->tris);
    free_ptr(d_->tri_info);
    free_ptr(d_->positions);
    free_ptr(d_->normals);
    free_ptr(d_->materials);
    free_ptr(d_->tri_light_pdf);
    free_ptr(d_->lights);
    free_ptr(d_->light_cdf);
    free_ptr(d_->e_table);
    Paths& p = d_->paths;
    free_ptr(p.ray_o);
    free_ptr(p.ray_d);
    free_ptr(p.hit_id);
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
    free_ptr(d_->queue[0]);
    free_ptr(d_->queue[1]);
    free_ptr(d_->shadow_queue);
    free_ptr(d_->transmit_queue);
    free_ptr(d_->counters);
    free_ptr(d_->film);
    free_ptr(d_->comp);
    free_ptr(d_->out);
    if (d_->stream) {
        cudaStreamDestroy(d_->stream);
    }
    cudaEventDestroy(d_->ev0);
    cudaEventDestroy(d_->ev1);
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
    uint32_t const nv = uint32_t(scene.positions.size() / 3);
    uint32_t const nt = uint32_t(scene.indices.size() / 3);
    if (nt == 0) {
        error_ = "scene has no triangles";
        return SPB_ERROR_STATE;
    }
    // Triangles of medium boundaries get their own class so shadow rays can pass them.
    std::vector<uint32_t> tri_class(nt, Class_surface);
    d_->has_media = false;
    for (uint32_t t = 0; t < nt; ++t) {
        if (scene.materials[scene.tri_material[t]].type == shading::Type_volume) {
            tri_class[t]  = Class_boundary;
            d_->has_media = true;
        }
    }
    Wide_bvh    bvh;
    std::string err;
    if (!build_wide_bvh(nv, nt, scene.positions.data(), scene.indices.data(), num_threads, bvh,
                        err, tri_class.data())) {
        error_ = "BVH build: " + err;
        return SPB_ERROR_ARGUMENT;
    }
    cudaDeviceSynchronize();
    SPB_RCUDA(upload(d_->nodes, bvh.nodes.data(), bvh.nodes.size() * sizeof(Wide_node)));
    SPB_RCUDA(upload(d_->tris, bvh.triangles.data(), bvh.triangles.size() * sizeof(Wide_triangle)));
    d_->hit_margin = bvh.hit_margin;

    std::vector<uint4> info(nt);
    for (uint32_t t = 0; t < nt; ++t) {
        info[t] = make_uint4(scene.indices[3 * t], scene.indices[3 * t + 1], scene.indices[3 * t + 2],
                             scene.tri_material[t]);
    }
    std::vector<float4> pos(nv), nrm(nv);
    for (uint32_t v = 0; v < nv; ++v) {
        pos[v] = make_float4(scene.positions[3 * v], scene.positions[3 * v + 1],
                             scene.positions[3 * v + 2], 0.f);
        nrm[v] = make_float4(scene.normals[3 * v], scene.normals[3 * v + 1], scene.normals[3 * v + 2],
                             0.f);
    }

    // Lights: every triangle of a light prop whose material emits, picked in proportion to
    // its power (area * mean radiance).
    std::vector<uint32_t> light_ids;
    std::vector<double>   power;
    std::vector<double>   area;
    for (uint32_t t = 0; t < nt; ++t) {
        shading::Material const& m = scene.materials[scene.tri_material[t]];
        if (!scene.tri_light[t] || m.type != shading::Type_light) {
            continue;
        }
        float const* a = &scene.positions[3 * scene.indices[3 * t]];
        float const* b = &scene.positions[3 * scene.indices[3 * t + 1]];
        float const* c = &scene.positions[3 * scene.indices[3 * t + 2]];
        double const e1[3] = {double(b[0]) - a[0], double(b[1]) - a[1], double(b[2]) - a[2]};
        double const e2[3] = {double(c[0]) - a[0], double(c[1]) - a[1], double(c[2]) - a[2]};
        double const cx = e1[1] * e2[2] - e1[2] * e2[1];
        double const cy = e1[2] * e2[0] - e1[0] * e2[2];
        double const cz = e1[0] * e2[1] - e1[1] * e2[0];
        double const ar = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
        double const pw = ar * (double(m.emission.x) + m.emission.y + m.emission.z) / 3.0;
        if (ar > 0.0 && pw > 0.0) {
            light_ids.push_back(t);
            power.push_back(pw);
            area.push_back(ar);
        }
    }
    double total = 0.0;
    for (double pw : power) {
        total += pw;
    }
    std::vector<float>  cdf(light_ids.size() + 1, 0.f);
    std::vector<float4> lights(3 * light_ids.size());
    std::vector<float>  tri_pdf(nt, 0.f);
    double run = 0.0;
    for (size_t l = 0; l < light_ids.size(); ++l) {
        uint32_t const t    = light_ids[l];
        double const   pick = power[l] / total;
        float const*   a    = &scene.positions[3 * scene.indices[3 * t]];
        float const*   b    = &scene.positions[3 * scene.indices[3 * t + 1]];
        float const*   c    = &scene.positions[3 * scene.indices[3 * t + 2]];
        lights[3 * l + 0]   = make_float4(a[0], a[1], a[2], float(area[l]));
        lights[3 * l + 1]   = make_float4(b[0] - a[0], b[1] - a[1], b[2] - a[2], float(pick));
        float4 e2           = make_float4(c[0] - a[0], c[1] - a[1], c[2] - a[2], 0.f);
        uint32_t tid        = t;
        std::memcpy(&e2.w, &tid, 4);
        lights[3 * l + 2]   = e2;
        run += pick;
        cdf[l + 1] = float(run);
        tri_pdf[t] = float(pick / area[l]);
    }
    if (!light_ids.empty()) {
        cdf.back() = 1.f;
    }
    d_->num_lights = uint32_t(light_ids.size());

    SPB_RCUDA(upload(d_->tri_info, info.data(), info.size() * sizeof(uint4)));
    SPB_RCUDA(upload(d_->positions, pos.data(), pos.size() * sizeof(float4)));
    SPB_RCUDA(upload(d_->normals, nrm.data(), nrm.size() * sizeof(float4)));
    SPB_RCUDA(upload(d_->materials, scene.materials.data(),
                     scene.materials.size() * sizeof(shading::Material)));
    SPB_RCUDA(upload(d_->tri_light_pdf, tri_pdf.data(), tri_pdf.size() * sizeof(float)));
    SPB_RCUDA(upload(d_->lights, lights.data(), lights.size() * sizeof(float4)));
    SPB_RCUDA(upload(d_->light_cdf, cdf.data(), cdf.size() * sizeof(float)));
    SPB_RCUDA(upload(d_->e_table, ggx_albedo_table(),
                     Ggx_table_size * Ggx_table_size * sizeof(float)));
    scene_ready_ = true;
    return SPB_OK;
}

int32_t Renderer::set_camera(Camera_desc const& camera) {
    if (camera.width == 0 || camera.height == 0 || !(camera.fov > 0.f)) {
        error_ = "camera needs a resolution and a field of view";
        return SPB_ERROR_ARGUMENT;
    }
    camera_ = camera;
    uint32_t const pixels = camera.width * camera.height;
    if (pixels != d_->film_pixels) {
        free_ptr(d_->film);
        free_ptr(d_->comp);
        free_ptr(d_->out);
        SPB_RCUDA(cudaMalloc(&d_->film, pixels * sizeof(float4)));
        SPB_RCUDA(cudaMalloc(&d_->comp, pixels * sizeof(float4)));
        SPB_RCUDA(cudaMalloc(&d_->out, pixels * sizeof(float4)));
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

int32_t Renderer::ensure_buffers(uint32_t paths) {
    if (paths <= d_->capacity) {
        return SPB_OK;
    }
    Paths& p = d_->paths;
    free_ptr(p.ray_o);
    free_ptr(p.ray_d);
    free_ptr(p.hit_id);
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
    free_ptr(d_->queue[0]);
    free_ptr(d_->queue[1]);
    free_ptr(d_->shadow_queue);
    free_ptr(d_->transmit_queue);
    size_t const n = paths;
    SPB_RCUDA(cudaMalloc(&p.ray_o, n * sizeof(float4)));
    SPB_RCUDA(cudaMalloc(&p.ray_d, n * sizeof(float4)));
    SPB_RCUDA(cudaMalloc(&p.hit_id, n * sizeof(uint32_t)));
    SPB_RCUDA(cudaMalloc(&p.hit_t, n * sizeof(float)));
    SPB_RCUDA(cudaMalloc(&p.hit_uv, n * sizeof(float2)));
    SPB_RCUDA(cudaMalloc(&p.T, n * sizeof(float4)));
    SPB_RCUDA(cudaMalloc(&p.L, n * sizeof(float4)));
    SPB_RCUDA(cudaMalloc(&p.puv, n * sizeof(float2)));
    SPB_RCUDA(cudaMalloc(&p.rng, n * sizeof(uint4)));
    SPB_RCUDA(cudaMalloc(&p.info, n * sizeof(uint32_t)));
    SPB_RCUDA(cudaMalloc(&p.sh_o, n * sizeof(float4)));
    SPB_RCUDA(cudaMalloc(&p.sh_d, n * sizeof(float4)));
    SPB_RCUDA(cudaMalloc(&p.sh_L, n * sizeof(float4)));
    SPB_RCUDA(cudaMalloc(&d_->queue[0], n * sizeof(uint32_t)));
    SPB_RCUDA(cudaMalloc(&d_->queue[1], n * sizeof(uint32_t)));
    SPB_RCUDA(cudaMalloc(&d_->shadow_queue, n * sizeof(uint32_t)));
    SPB_RCUDA(cudaMalloc(&d_->transmit_queue, n * sizeof(uint32_t)));
    if (!d_->counters) {
        SPB_RCUDA(cudaMalloc(&d_->counters, Counter_words * sizeof(uint32_t)));
    }
    d_->capacity = paths;
    return SPB_OK;
}

int32_t Renderer::render(uint32_t first_sample, uint32_t num_samples) {
    if (!ready()) {
        error_ = "render needs a scene and a camera";
        return SPB_ERROR_STATE;
    }
    if (settings_.max_bounces + 2 > Max_bounce_slots) {
        error_ = "max_bounces too large";
        return SPB_ERROR_ARGUMENT;
    }
    uint32_t const pixels = camera_.width * camera_.height;
    // k samples per pixel per wave, up to about 4M paths per wave.
    uint32_t const per_wave = std::max(1u, std::min(num_samples, (1u << 22) / std::max(1u, pixels)));
    if (int32_t const st = ensure_buffers(per_wave * pixels)) {
        return st;
    }

    float const ratio = float(camera_.height) / float(camera_.width);
    float const z     = 1.f / std::tan(0.5f * camera_.fov);
    Cam         cam;
    cam.left_top = make_float3(-1.f, ratio, z);
    cam.d_x      = make_float3(2.f / float(camera_.width), 0.f, 0.f);
    cam.d_y      = make_float3(0.f, -2.f * ratio / float(camera_.height), 0.f);
    cam.r0       = make_float3(camera_.rotation[0], camera_.rotation[1], camera_.rotation[2]);
    cam.r1       = make_float3(camera_.rotation[3], camera_.rotation[4], camera_.rotation[5]);
    cam.r2       = make_float3(camera_.rotation[6], camera_.rotation[7], camera_.rotation[8]);
    cam.pos      = make_float3(camera_.position[0], camera_.position[1], camera_.position[2]);
    cam.w        = camera_.width;
    cam.h        = camera_.height;

    Scene_gpu sg;
    sg.nodes         = d_->nodes;
    sg.tris          = d_->tris;
    sg.hit_margin    = d_->hit_margin;
    sg.tri_info      = d_->tri_info;
    sg.positions     = d_->positions;
    sg.normals       = d_->normals;
    sg.materials     = d_->materials;
    sg.tri_light_pdf = d_->tri_light_pdf;
    sg.lights        = d_->lights;
    sg.light_cdf     = d_->light_cdf;
    sg.num_lights    = d_->num_lights;
    sg.e_table       = d_->e_table;

    cudaStream_t const st = d_->stream;
    uint32_t* const    ctr = d_->counters;
    uint32_t const     bounces = settings_.max_bounces + 1;

    stats_ = Stats();
    std::vector<uint32_t> host_ctr(Counter_words);
    SPB_RCUDA(cudaEventRecord(d_->ev0, st));
    for (uint32_t done = 0; done < num_samples;) {
        uint32_t const k     = std::min(per_wave, num_samples - done);
        uint32_t const paths = k * pixels;
        Wave           wave{first_sample + done, k, settings_.seed, settings_.min_bounces,
                  settings_.max_bounces};
        SPB_RCUDA(cudaMemsetAsync(ctr, 0, Counter_words * sizeof(uint32_t), st));
        k_generate<<<(paths + 255) / 256, 256, 0, st>>>(cam, wave, d_->paths, d_->queue[0], ctr,
                                                         paths);
        for (uint32_t b = 0; b < bounces; ++b) {
            uint32_t* const q_in  = d_->queue[b & 1];
            uint32_t* const q_out = d_->queue[(b + 1) & 1];
            uint32_t* const c = ctr + Counter_stride * b;
            k_trace<false><<<d_->trace_grid, Trace_block, 0, st>>>(sg, d_->paths, q_in, c, c + 2,
                                                                   ctr + Overflow_slot);
            k_shade<<<(paths + Shade_block - 1) / Shade_block, Shade_block, 0, st>>>(
                sg, wave, d_->paths, q_in, c, q_out, c + Counter_stride, d_->shadow_queue, c + 1);
            if (d_->has_media) {
                k_trace<true, true><<<d_->trace_grid, Trace_block, 0, st>>>(
                    sg, d_->paths, d_->shadow_queue, c + 1, c + 3, ctr + Overflow_slot,
                    d_->transmit_queue, c + 4);
                k_transmit<<<(paths + Trace_block - 1) / Trace_block, Trace_block, 0, st>>>(
                    sg, d_->paths, d_->transmit_queue, c + 4, ctr + Overflow_slot);
            } else {
                k_trace<true><<<d_->trace_grid, Trace_block, 0, st>>>(
                    sg, d_->paths, d_->shadow_queue, c + 1, c + 3, ctr + Overflow_slot);
            }
        }
        k_gather<<<(pixels + 255) / 256, 256, 0, st>>>(d_->paths, camera_.width, camera_.height, k,
                                                      d_->film, d_->comp);
        SPB_RCUDA(cudaGetLastError());
        SPB_RCUDA(cudaMemcpyAsync(host_ctr.data(), ctr, Counter_words * sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, st));
        SPB_RCUDA(cudaStreamSynchronize(st));
        for (uint32_t b = 0; b < bounces; ++b) {
            stats_.extension_rays += host_ctr[Counter_stride * b];
            stats_.shadow_rays += host_ctr[Counter_stride * b + 1];
        }
        stats_.overflow += host_ctr[Overflow_slot];
        stats_.paths += paths;
        done += k;
    }
    SPB_RCUDA(cudaEventRecord(d_->ev1, st));
    SPB_RCUDA(cudaEventSynchronize(d_->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, d_->ev0, d_->ev1);
    stats_.seconds = double(ms) * 1e-3;
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
