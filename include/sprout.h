/*
 * sprout C API, served by the B200 path tracer in libsprout_b200.so.
 *
 * Same entry points, signatures and return codes as the reference's C API
 * (source/capi/sprout.h:39-122, implemented in source/capi/capi.cpp:133-750), so a program
 * written against the reference's libsprout.so runs unchanged when it loads this library
 * instead.  Codes: 0 ok, -1 no engine / bad argument, -2 invalid state; id-returning calls
 * return SU_RESOURCE_NULL (0xFFFFFFFF) on failure.  Messages go to the su_register_log
 * callback.
 *
 * Scope of this implementation (the rendering hot path): perspective camera, triangle meshes
 * (indexed, with normals, optional parts; in memory or from mesh JSON files), the built-in
 * Cube, Disk, Rectangle, Sphere and Infinite_sphere shapes, the Substitute (Disney + GGX),
 * Light (constant emission) and Volumetric (homogeneous or density-grid) materials, mesh and
 * environment lights, one-channel images as density grids, take and scene files through
 * su_load_take / su_mount, the PTMIS integrator (with optional path guiding), progressive and
 * batch rendering, framebuffer readout and the default PNG export.  The Canopy,
 * Distant_sphere and Plane shapes and animation frames return -2 / SU_RESOURCE_NULL with a
 * logged reason.  Each declaration below cites the reference function it replaces.
 *
 * Deviation: su_copy_framebuffer(SU_FLOAT32, ..., 4, ...) returns 0 after copying; the
 * reference copies and then returns -2 (capi.cpp:704-714).
 */
#ifndef SPROUT_B200_SU_H
#define SPROUT_B200_SU_H

#include <stdbool.h>
#include <stdint.h>

#if defined(_WIN32)
#define SU_LIBRARY_API __declspec(dllexport)
#else
#define SU_LIBRARY_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SU_RESOURCE_NULL 0xFFFFFFFF

#define SU_SHAPE_CANOPY 0
#define SU_SHAPE_CUBE 1
#define SU_SHAPE_DISK 2
#define SU_SHAPE_DISTANT_SPHERE 3
#define SU_SHAPE_INFINITE_SPHERE 4
#define SU_SHAPE_PLANE 5
#define SU_SHAPE_RECTANGLE 6
#define SU_SHAPE_SPHERE 7

#define SU_UINT8 0
#define SU_FLOAT32 2

#define SU_LOG_INFO 0
#define SU_LOG_WARNING 1
#define SU_LOG_ERROR 2
#define SU_LOG_VERBOSE 3

/* capi.cpp:133-135 */
SU_LIBRARY_API char const* su_platform_revision(void);
/* capi.cpp:137-147: creates the single engine; -1 if one exists */
SU_LIBRARY_API int32_t su_init(bool progressive);
/* capi.cpp:149-154 */
SU_LIBRARY_API int32_t su_release(void);
/* capi.cpp:156-162: folders searched (last mounted first) for files named by takes, scenes and the *_from_file calls */
SU_LIBRARY_API int32_t su_mount(char const* folder);
/* capi.cpp:164-173 */
SU_LIBRARY_API int32_t su_clear(void);
/* capi.cpp:175-206: a take as JSON text or a file name (camera, sampler, integrator, scene file with
   materials and Prop / Light entities); -2 if it cannot be read or names something unsupported */
SU_LIBRARY_API int32_t su_load_take(char const* string);
/* capi.cpp:208-229 */
SU_LIBRARY_API int32_t su_create_defaults(void);
/* capi.cpp:231-243: {"Perspective": {"parameters": {"fov": degrees}}, "resolution"} subset */
SU_LIBRARY_API uint32_t su_create_camera(char const* string);
/* capi.cpp:245-276 */
SU_LIBRARY_API uint32_t su_create_camera_perspective(uint32_t width, uint32_t height, float fov);
/* capi.cpp:278-291 */
SU_LIBRARY_API int32_t su_camera_set_resolution(uint32_t width, uint32_t height);
/* capi.cpp:293-312 */
SU_LIBRARY_API int32_t su_create_sampler(uint32_t num_samples);
/* capi.cpp:314-326: {"surface": {"PTMIS": {"min_bounces", "max_bounces"}}} */
SU_LIBRARY_API int32_t su_create_integrators(char const* string);
/* capi.cpp:328-345: one-channel float or byte images (2-D or 3-D), used as density grids by Volumetric
   materials; other channel counts return SU_RESOURCE_NULL */
SU_LIBRARY_API uint32_t su_create_image(uint32_t pixel_type, uint32_t num_channels, uint32_t width,
                                        uint32_t height, uint32_t depth, uint32_t num_elements,
                                        uint32_t stride, char const* data);
/* capi.cpp:347-365: {"rendering": {"Substitute" | "Light" | "Volumetric": {...}}} */
SU_LIBRARY_API uint32_t su_create_material(char const* string);
/* capi.cpp:367-376: a material JSON file (as su_create_material), under the mounted folders first */
SU_LIBRARY_API uint32_t su_create_material_from_file(char const* filename);
/* capi.cpp:378-406 (the mesh is copied at call time) */
SU_LIBRARY_API uint32_t su_create_triangle_mesh_async(
    uint32_t num_triangles, uint32_t num_vertices, uint32_t positions_stride,
    float const* positions, uint32_t normals_stride, float const* normals, uint32_t tangents_stride,
    float const* tangents, uint32_t uvs_stride, float const* uvs, uint32_t const* indices,
    uint32_t num_parts, uint32_t const* parts);
/* capi.cpp:408-418: a triangle-mesh JSON file, under the mounted folders first */
SU_LIBRARY_API uint32_t su_create_triangle_mesh_from_file(char const* filename);
/* capi.cpp:420-451 */
SU_LIBRARY_API uint32_t su_create_prop(uint32_t shape, uint32_t num_materials,
                                       uint32_t const* materials);
/* capi.cpp:453-463 */
SU_LIBRARY_API int32_t su_create_light(uint32_t entity);
/* capi.cpp:465-473 */
SU_LIBRARY_API uint32_t su_camera_entity(void);
/* capi.cpp:475-488 */
SU_LIBRARY_API int32_t su_camera_sensor_dimensions(int32_t* dimensions);
/* capi.cpp:490-500: animation frames are out of scope: returns -2 */
SU_LIBRARY_API int32_t su_entity_allocate_frames(uint32_t entity);
/* capi.cpp:502-514 */
SU_LIBRARY_API int32_t su_entity_transformation(uint32_t entity, float* trafo);
/* capi.cpp:516-537: row-major 4x4 object-to-world, translation in the last row */
SU_LIBRARY_API int32_t su_entity_set_transformation(uint32_t entity, float const* trafo);
/* capi.cpp:539-563: returns -2 (animation out of scope) */
SU_LIBRARY_API int32_t su_entity_set_transformation_frame(uint32_t entity, uint32_t frame,
                                                          float const* trafo);
/* capi.cpp:565-580 */
SU_LIBRARY_API int32_t su_render(void);
/* capi.cpp:582-596 */
SU_LIBRARY_API int32_t su_render_frame(uint32_t frame);
/* capi.cpp:598-604: writes output_NNNNNN.png (8-bit sRGB) into the working directory */
SU_LIBRARY_API int32_t su_export_frame(uint32_t frame);
/* capi.cpp:606-624 */
SU_LIBRARY_API int32_t su_start_render_frame(uint32_t frame);
/* capi.cpp:626-632 */
SU_LIBRARY_API int32_t su_set_expected_iterations(uint32_t iterations);
/* capi.cpp:634-646 */
SU_LIBRARY_API int32_t su_render_iteration(void);
/* capi.cpp:648-656 */
SU_LIBRARY_API int32_t su_postprocess(void);
/* capi.cpp:658-715 */
SU_LIBRARY_API int32_t su_copy_framebuffer(uint32_t type, uint32_t width, uint32_t height,
                                           uint32_t num_channels, uint8_t* destination);

typedef void (*Post)(uint32_t type, char const* text);
/* capi.cpp:733-741 */
SU_LIBRARY_API int32_t su_register_log(Post post);

typedef void (*Progress_start)(uint32_t resolution);
typedef void (*Progress_tick)(void);
/* capi.cpp:743-750 */
SU_LIBRARY_API int32_t su_register_progress(Progress_start start, Progress_tick tick);

#ifdef __cplusplus
}
#endif

#endif
