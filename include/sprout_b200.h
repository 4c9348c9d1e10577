/*
 * sprout_b200 — C ABI of the B200 ray-cast path (closest hit / any hit over an SAH BVH).
 *
 * This library replaces the reference's per-ray triangle-mesh traversal with a batched
 * GPU cast.  Each entry point names the reference interface it stands in for
 * (paths are relative to the reference project, Opioid/sprout).
 *
 * Conventions
 *   - Every function returns int32_t: 0 on success, SPB_ERROR_ARGUMENT (-1) for a bad
 *     argument (null pointer, size out of range), SPB_ERROR_STATE (-2) for a call that is
 *     not valid in the object's current state (e.g. casting before a build), and
 *     SPB_ERROR_CUDA (-3) when a CUDA call fails.  These mirror the reference capi's codes
 *     (source/capi/capi.cpp:112-131: -1 no engine / bad argument, -2 invalid state).
 *     spb_last_error() returns a readable message for the last failure on this thread.
 *   - A ray is 8 floats, exactly the reference's math::ray storage order
 *     (source/base/math/ray.hpp:8-28, ray.inl:11-16): origin.xyz, min_t, direction.xyz,
 *     max_t.  Rays are read-only.
 *   - Results are per ray: the caller's triangle index of the closest hit
 *     (SPB_MISS = 0xFFFFFFFF for no hit), the hit distance t (the ray's max_t after the
 *     call: the hit t, or the unchanged max_t on a miss, as the reference leaves
 *     ray.max_t()), and optionally the barycentrics u, v of the hit.
 *   - "_device" entry points take device pointers and a cudaStream_t (passed as void*,
 *     NULL = the legacy default stream) and are asynchronous with respect to the host.
 *     "_host" entry points take host pointers (pinned or pageable), copy the rays to the
 *     GPU in chunks, cast, copy the results back and return when they are in host memory.
 *   - Calls on one tree must not overlap on the GPU (they share the tree's work counter):
 *     issue them on one stream, or synchronize between streams.  Different trees are
 *     independent.  Like the reference engine, a tree object is not re-entrant from
 *     several host threads.
 */
#ifndef SPROUT_B200_H
#define SPROUT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define SPB_API __declspec(dllexport)
#else
#define SPB_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SPB_OK 0
#define SPB_ERROR_ARGUMENT -1
#define SPB_ERROR_STATE -2
#define SPB_ERROR_CUDA -3

#define SPB_MISS 0xFFFFFFFFu

/* Largest batch one call accepts (ray indices are 32-bit on the device). */
#define SPB_MAX_RAYS_PER_CALL 0x7FFFFFFFull

typedef struct spb_tree spb_tree;

typedef struct spb_tree_info {
    uint32_t num_triangles;   /* triangles given to spb_tree_build */
    uint32_t num_nodes;       /* 8-wide nodes (80 bytes each) */
    uint32_t num_leaves;      /* leaf slots (1-3 triangles each) */
    uint32_t max_depth;       /* deepest node, root = 1 */
    uint64_t device_bytes;    /* nodes + triangles resident on the device */
    double   build_seconds;   /* host build + upload time of the last build */
    double   sah_cost;        /* SAH cost of the 8-wide tree (traversal 1, triangle 1) */
} spb_tree_info;

/* Readable message for the last error on the calling thread ("" if none). */
SPB_API char const* spb_last_error(void);

/* Library version string. */
SPB_API char const* spb_version(void);

/*
 * Create / release a tree bound to the current CUDA device.
 * Replaces constructing scene::shape::triangle::bvh::Tree
 * (source/core/scene/shape/triangle/bvh/triangle_bvh_tree.cpp:15-20).
 */
SPB_API int32_t spb_tree_create(spb_tree** tree);
SPB_API int32_t spb_tree_release(spb_tree* tree);

/*
 * Build the BVH over an indexed triangle mesh and upload it.
 * positions: num_vertices * 3 floats (host); indices: num_triangles * 3 uint32 (host).
 * Replaces bvh::Builder_SAH(16, 64, 4).build(tree, ...)
 * (source/core/scene/shape/triangle/triangle_mesh_provider.cpp:375-378,
 *  source/core/scene/shape/triangle/bvh/triangle_bvh_builder_sah.cpp:21-67).
 * num_threads: host build threads (0 = all hardware threads).
 */
SPB_API int32_t spb_tree_build(spb_tree* tree, uint32_t num_vertices, uint32_t num_triangles,
                               float const* positions, uint32_t const* indices,
                               uint32_t num_threads);

SPB_API int32_t spb_tree_info_get(spb_tree const* tree, spb_tree_info* info);

/*
 * Closest hit for a batch of rays (device pointers).
 * Replaces Tree::intersect (source/core/scene/shape/triangle/bvh/triangle_bvh_tree.cpp:41-90)
 * called once per ray.  ids and ts are required; uvs (2 floats per ray) may be NULL.
 */
SPB_API int32_t spb_intersect_device(spb_tree* tree, float const* rays, uint64_t num_rays,
                                     uint32_t* ids, float* ts, float* uvs, void* stream);

/*
 * Any hit (occlusion) for a batch of rays (device pointers): occluded[i] = 1 if some
 * triangle is hit with min_t <= t <= max_t, else 0.
 * Replaces Tree::intersect_p (source/core/scene/shape/triangle/bvh/triangle_bvh_tree.cpp:145-185).
 */
SPB_API int32_t spb_intersect_p_device(spb_tree* tree, float const* rays, uint64_t num_rays,
                                       uint8_t* occluded, void* stream);

/* Host-memory forms of the two calls above (copies and cast pipelined over streams). */
SPB_API int32_t spb_intersect_host(spb_tree* tree, float const* rays, uint64_t num_rays,
                                   uint32_t* ids, float* ts, float* uvs);
SPB_API int32_t spb_intersect_p_host(spb_tree* tree, float const* rays, uint64_t num_rays,
                                     uint8_t* occluded);

/*
 * Closest hit (device pointers, as spb_intersect_device) that also counts the traversal's
 * work: node_steps receives the 8-wide nodes visited and triangle_steps the triangles tested,
 * summed over all rays of the batch.  Synchronizes the stream before returning the counts.
 * For measurement (bytes fetched per ray: nodes x 80 + triangles x 48); the counting costs
 * a few percent, so timed casts use spb_intersect_device.  The reference counts nothing of
 * the kind; its Tree::intersect (source/core/scene/shape/triangle/bvh/triangle_bvh_tree.cpp:41-90)
 * visits nodes and tests triangles in the same sense.
 */
SPB_API int32_t spb_cast_stats_device(spb_tree* tree, float const* rays, uint64_t num_rays,
                                      uint32_t* ids, float* ts, void* stream,
                                      uint64_t* node_steps, uint64_t* triangle_steps);

/*
 * Device-side status of the casts on this tree: number of rays whose traversal stack would
 * have overflowed, counted over every cast entry point since the tree was created (always 0
 * for trees this library builds; the kernel checks and drops such rays as misses instead of
 * writing out of bounds).  Synchronizes the device.
 */
SPB_API int32_t spb_tree_status(spb_tree* tree, uint32_t* overflowed_rays);

/*
 * Synthetic inputs of the cast benchmark (deterministic, host memory).
 *
 * spb_synth_sphere_mesh: a tetrahedron whose faces are subdivided n x n, projected to the
 * unit sphere and displaced radially by amplitude * fBm (6 octaves, lacunarity 2, gain 0.5,
 * gradient noise seeded by seed).  4 n^2 triangles, 2 n^2 + 2 vertices; every vertex has
 * valence <= 6.  Pass NULL buffers to query the sizes only.
 *
 * spb_synth_rays: ray i (i = first .. first + count - 1) draws from a PCG32 stream
 * (sequence i, state seed): origin uniform in [-extent, extent]^3, direction uniform on the
 * unit sphere, min_t = 0, max_t = 3.4027715e38 (the reference's scene::Ray_max_t,
 * source/core/scene/scene_constants.hpp:10).
 */
SPB_API int32_t spb_synth_sphere_mesh(uint32_t n, float amplitude, uint32_t seed,
                                      uint32_t* num_vertices, uint32_t* num_triangles,
                                      float* positions, uint32_t* indices);
SPB_API int32_t spb_synth_rays(uint64_t first, uint64_t count, uint32_t seed, float extent,
                               float* rays, uint32_t num_threads);

/*
 * Closest hit without any device allocation: rays and results in host memory, staged through
 * a fixed device array that the library reserves when it is loaded.  No counterpart in the
 * reference (its CPU cast allocates nothing on a GPU).  It is for callers that cannot call
 * cudaMalloc: a cudaMalloc may synchronize the device and may fail when device memory runs
 * out, so a frame loop with a fixed time budget, or an application whose own allocator owns
 * all device memory, must not allocate per call -- spb_intersect_host allocates staging
 * buffers on its first call, this entry point never does.
 *
 * Limit: at most SPB_STATIC_MAX_RAYS rays per call (larger batches are rejected with
 * SPB_ERROR_ARGUMENT); the fixed array (SPB_STATIC_MAX_RAYS * 40 bytes + 256 bytes, about
 * 2.5 MiB) stays allocated on every GPU that loads the library until the process exits.
 * The first call on a device looks up the array's device address (once per device).
 * The address is looked up again in a new CUDA context (after a cudaDeviceReset, say).
 * All calls share the one array, so calls that overlap on the GPU -- from several host
 * threads, or on several trees at once -- race and must be serialized by the caller.
 * Results are identical to spb_intersect_host, and so is the error behaviour: rays that
 * would overflow the traversal stack (none for trees this library builds) end as misses and
 * are counted where spb_tree_status reports them.  Uses the legacy default stream and returns
 * when the results are in host memory.
 */
#define SPB_STATIC_MAX_RAYS 65536ull
SPB_API int32_t spb_intersect_host_static(spb_tree* tree, float const* rays, uint64_t num_rays,
                                          uint32_t* ids, float* ts);

/*
 * Counters of the path tracer's last su_render / su_render_frame / su_render_iteration call
 * (the su_* engine of include/sprout.h): camera samples traced, closest-hit rays (camera and
 * continuation), any-hit (shadow) rays, and the device time between the first and last
 * kernel.  With path guiding: the vertices the network was evaluated for and the device time
 * of that inference (input encoding included), and the training samples (Adam steps x batch)
 * and the device time of training (batch gathering, gradients, Adam).  Launch shapes: the
 * largest wave (paths) and the traversal blocks per SM of the last wave, as the autotuner (or
 * the integrator's "wave_paths" / "trace_blocks_per_sm" keys) set them, and the waves replayed
 * from captured CUDA graphs (the "cuda_graphs" key turns them off).  Scene: the props kept
 * as instances of shared per-mesh trees under a top-level tree (the "instancing" key; 0 when
 * every prop was flattened into one tree), the triangles the uploaded trees hold, and the
 * medium tracking segments that reached the 65,536-collision cap.  No counterpart in the
 * reference (it logs wall-clock phases only, rendering_driver.cpp:99-136).
 * SPB_ERROR_ARGUMENT if there is no engine.
 */
typedef struct spb_render_stats {
    uint64_t paths;
    uint64_t extension_rays;
    uint64_t shadow_rays;
    double   device_seconds;
    uint32_t overflow;
    uint64_t guide_vertices;
    double   guide_inference_seconds;
    uint64_t guide_training_samples;
    double   guide_training_seconds;
    uint32_t wave_paths;
    uint32_t trace_blocks_per_sm;
    uint32_t graph_waves;
    uint32_t instances;         /* props under a top-level tree (0: the scene was flattened) */
    uint32_t tracking_capped;   /* medium tracking segments cut at the step cap (0 expected) */
    uint64_t device_triangles;  /* triangles in the uploaded trees */
} spb_render_stats;
SPB_API int32_t spb_render_last_stats(spb_render_stats* out);

/*
 * Several views of the engine's scene in one render: the scene the su_* calls built (uploaded
 * first if it changed), the integrator, sampler kind and settings of the engine, and `count`
 * cameras, each with its own resolution, horizontal field of view (radians) and row-major
 * 4 x 4 camera-to-world transformation (as su_entity_set_transformation takes for the camera
 * entity).  Every view gets samples_per_pixel samples; their paths share the renderer's waves,
 * so small views fill the GPU together, and each view traces the same paths as when rendered
 * alone.  rgba receives the resolved linear images one after another (view 0's
 * width x height x 4 floats first), as su_copy_framebuffer(SU_FLOAT32, ...) would for each.
 * No counterpart in the reference, which renders one camera per frame (rendering_driver.cpp);
 * the engine's own camera is re-applied by its next su_* frame.
 * SPB_ERROR_STATE without an engine or complete scene, SPB_ERROR_ARGUMENT for bad views
 * (1 to 4096 of them, each with a positive resolution and field of view).
 */
typedef struct spb_view {
    uint32_t width;
    uint32_t height;
    float    fov;
    float    transformation[16];
} spb_view;
SPB_API int32_t spb_render_views(uint32_t count, spb_view const* views, uint32_t samples_per_pixel,
                                 float* rgba);

/*
 * The 32 x 32 GGX directional-albedo table the Substitute material's energy compensation
 * reads (row = alpha index, column = cos(theta_o) index, both i / 31), as computed by this
 * library.  Stands in for the reference's generated table E
 * (source/core/scene/material/ggx/ggx_integral.inl, generator ggx_integrate.cpp:199-230).
 * out: 1024 floats.
 */
SPB_API int32_t spb_ggx_albedo_table(float* out);

/*
 * Path guiding (no counterpart in the reference, which has no path guiding).  The renderer's
 * guiding network maps a 32-float encoding of a path vertex (position, normal, outgoing
 * direction) through four hidden layers of 64 (ReLU) to 40 outputs: eight von Mises-Fisher
 * lobes (unnormalised mean direction, log-concentration) and eight mixture logits.  Its
 * parameters are packed per layer as W (outputs x inputs, row-major) then b; the products run
 * with BF16 operands and FP32 accumulation.  These entry points expose the network's forward
 * pass and its training gradient on host arrays, so that both can be checked against a CPU
 * restatement.
 *
 * spb_guide_parameter_count: the packed parameter count (17,192).
 * spb_guide_forward: outputs (n x 40) for inputs (n x 32).
 * spb_guide_gradients: gradient (parameter count) of (1/n) sum_i weights[i] * (-log q_i),
 *   q_i the mixture's density at directions[i] (n x 3, unit vectors) for inputs[i].
 */
SPB_API int32_t spb_guide_parameter_count(uint32_t* count);
SPB_API int32_t spb_guide_forward(float const* params, float const* inputs, uint64_t n, float* outputs);
SPB_API int32_t spb_guide_gradients(float const* params, float const* inputs, float const* directions,
                                    float const* weights, uint64_t n, float* gradient);

#ifdef __cplusplus
}
#endif

#endif
