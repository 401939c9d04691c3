/*
 * rtc.h - C ABI of the B200-native path-tracing hot path.
 *
 * This is the drop-in boundary for the render call of flarive/CortexRaytracerCuda:
 *
 *   void launchGPU(const sceneConfig& cfg, int width, int height, int spp, int max_depth,
 *                  int tx, int ty, const char* filepath, bool quietMode)
 *     (core/src/gpu.cu:2127, declared core/src/renderers/gpu_cuda_renderer.h:17)
 *
 * reached through the virtual renderer::render(const sceneConfig&, const render_parameters&)
 * (core/src/renderers/renderer.h:16).  Every entry point takes plain pointers and sizes, returns
 * an rtc_status and never exits the process (the reference prints and calls exit(99),
 * core/src/gpu.cu:119-129).
 *
 * Scene model.  A scene is a flat POD description (rtc_scene_desc) with 32-bit counts, replacing the
 * reference's sceneConfig tree with uint8_t counts (core/src/scenes/scene_config.h:394-459).  Objects
 * get a global primitive id in the order the reference's load_scene adds them to its world list
 * (core/src/gpu.cu:504-635): directional lights, then spheres, then quads, then mesh triangles (mesh
 * by mesh, triangle by triangle).  Materials and textures are referenced by index instead of by name
 * (the reference matches names with strcmp_device, core/src/gpu.cu:132).
 *
 * Pixel layout.  Radiance buffers use the reference's frame-buffer order: pixel (i, j) with j counted
 * from the BOTTOM row is element j*width + i (core/src/gpu.cu:769).  The 8-bit RGB output is in PNG
 * order (top row first), i.e. the rows are flipped as the reference's host loop does
 * (core/src/gpu.cu:2098-2107).
 */
#ifndef RTC_H
#define RTC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------------ */
/* status                                                                                            */
/* ------------------------------------------------------------------------------------------------ */

typedef enum rtc_status {
    RTC_OK = 0,
    RTC_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, bad enum value                       */
    RTC_ERR_BAD_SCENE = 2,        /* scene references a missing material/texture/image, NaN coords */
    RTC_ERR_CUDA = 3,             /* a CUDA runtime call failed; see rtc_last_error_string()       */
    RTC_ERR_OOM = 4,              /* device allocation failed or the HBM budget would be exceeded  */
    RTC_ERR_TIMEOUT = 5,          /* a bounded device-side wait ran out                            */
    RTC_ERR_NO_DEVICE = 6,        /* no CUDA device, or the device is not sm_100                   */
    RTC_ERR_IO = 7,               /* file could not be written / read                               */
    RTC_ERR_DEVICE_CHECK = 8,     /* a kernel's own bounds check fired (status word non-zero)      */
    RTC_ERR_NOT_FOUND = 9,        /* unknown handle / request id                                    */
    RTC_ERR_BUSY = 10             /* request still in flight                                        */
} rtc_status;

/* Text of the last error raised on the calling thread ("" when none). */
const char* rtc_last_error_string(void);

/* ------------------------------------------------------------------------------------------------ */
/* scene description                                                                                 */
/* ------------------------------------------------------------------------------------------------ */

/* Textures (core/src/textures/). */
typedef enum rtc_texture_kind {
    RTC_TEX_SOLID = 0,   /* solid_color_texture::value (solid_color_texture.cuh:34)                  */
    RTC_TEX_CHECKER = 1, /* checker_texture::value, spatial floor(p/scale) parity (checker_texture.cuh:33-41) */
    RTC_TEX_IMAGE = 2    /* image_texture::value, nearest RGB8 with V flip (image_texture.cuh:54-70)  */
} rtc_texture_kind;

typedef struct rtc_texture {
    int32_t kind;     /* rtc_texture_kind                                                            */
    float color[3];   /* SOLID: the colour                                                           */
    float scale;      /* CHECKER: cell size; the reference stores inv_scale = 1/scale               */
    int32_t even;     /* CHECKER: texture used where the cell parity is even (checker m_even)       */
    int32_t odd;      /* CHECKER: texture used where the parity is odd (checker m_odd)              */
    int32_t image;    /* IMAGE: index into rtc_scene_desc.images                                    */
} rtc_texture;

/* 8-bit RGB image, row-major, top row first (stbi_load order, core/src/gpu.cu:1743). */
typedef struct rtc_image {
    const uint8_t* rgb;
    int32_t width;
    int32_t height;
} rtc_image;

/* Materials (core/src/materials/). */
typedef enum rtc_material_kind {
    RTC_MAT_LAMBERTIAN = 0,    /* lambertian.cuh:63-143, mixture-PDF importance sampling         */
    RTC_MAT_METAL = 1,         /* metal.cuh:52-64                                                */
    RTC_MAT_DIELECTRIC = 2,    /* dielectric.cuh:32-63                                           */
    RTC_MAT_DIFFUSE_LIGHT = 3  /* diffuse_light.cuh:45-67, emits, never scatters                 */
} rtc_material_kind;

typedef struct rtc_material {
    int32_t kind;        /* rtc_material_kind                                                      */
    int32_t texture;     /* albedo (lambertian, metal) or emission (diffuse light) texture index   */
    float fuzz;          /* METAL: fuzz; values >= 1 are clamped to 1 as metal::metal does         */
    float ior;           /* DIELECTRIC: index of refraction                                        */
    float intensity;     /* DIFFUSE_LIGHT: emission scale                                          */
    int32_t directional; /* DIFFUSE_LIGHT: one-sided; back face emits RGBA(0,0,0,0)                */
} rtc_material;

/* Sphere (core/src/primitives/sphere.cuh). */
typedef struct rtc_sphere {
    float center[3];
    float radius;
    int32_t material;
} rtc_sphere;

/* Quad, lower-left corner q and edges u, v (core/src/primitives/quad.cuh). */
typedef struct rtc_quad {
    float q[3];
    float u[3];
    float v[3];
    int32_t material;
} rtc_quad;

/* Directional (quad) light centred on position (core/src/lights/directional_light.cuh).  It gets
 * its own diffuse_light(color, intensity, directional=true, invisible) material, and it is the only
 * kind of object that enters the light list sampled by the lambertian mixture PDF
 * (core/src/gpu.cu:681-694). */
typedef struct rtc_dir_light {
    float position[3];
    float u[3];
    float v[3];
    float color[3];
    float intensity;
    int32_t invisible;   /* hidden to primary rays: directional_light.cuh:106 */
} rtc_dir_light;

/* Omni light (omni_light, lights/omni_light.cuh): an emitting sphere; diffuse_light material that
 * emits color * intensity from both faces; sampled by solid angle (random_to_sphere); hidden to primary
 * rays when invisible. */
typedef struct rtc_omni_light {
    float position[3];
    float radius;
    float color[3];
    float intensity;
    int32_t invisible;
} rtc_omni_light;

/* Spot light (spot_light, lights/spot_light.cuh, with diffuse_spot_light, materials/
 * diffuse_spot_light.cuh): an emitting sphere whose front faces emit color * intensity *
 * cos^falloff toward rays within `cutoff` degrees of `direction` (and white outside it, as the
 * reference does); sampled like an omni light. */
typedef struct rtc_spot_light {
    float position[3];
    float direction[3];
    float cutoff;        /* degrees */
    float falloff;       /* exponent */
    float intensity;
    float radius;
    float color[3];
    int32_t invisible;
} rtc_spot_light;

/* Indexed triangle mesh; each triangle becomes one reference `triangle` (triangle.cuh:87-185). */
typedef struct rtc_mesh {
    const float* vertices;      /* 3 floats per vertex                                             */
    const uint32_t* indices;    /* 3 per triangle                                                  */
    const float* normals;       /* optional, 3 floats per vertex; used when smooth != 0            */
    const float* uvs;           /* optional, 2 floats per vertex: texture coordinates, interpolated at
                                   the hit with get_triangle_uv's barycentrics and wrapped into [0, 1)
                                   (uvmapping.cuh:415-447; the reference evaluates them at the hit
                                   record's previous hit point, triangle.cuh:162 - not reproduced)  */
    uint32_t num_vertices;
    uint32_t num_triangles;
    int32_t material;
    int32_t smooth;             /* barycentric normal interpolation (triangle.cuh:171-175)         */
} rtc_mesh;

/* Object transform, as scene_factory::applyTransform wraps a primitive (core/src/scene_factory.cuh:
 * 710-725): rt::translate inside, then rt::rotate, then rt::scale outside (primitives/translate.cuh,
 * rotate.cuh, scale.cuh).  A ray reaches the object through scale (o / s, d / s), rotate (the glm
 * matrix of -x, -y, -z degrees about x, then y, then z) and translate (o - t); the hit point returns
 * through translate (+ t), rotate (the matrix of +x, +y, +z degrees, which is not the inverse of the
 * first when two axes turn, as in the reference) and scale (p * s, normal unit(n / s)).  Only the parts
 * whose flag is set apply. */
#define RTC_XF_TRANSLATE 1u
#define RTC_XF_ROTATE 2u
#define RTC_XF_SCALE 4u
typedef struct rtc_transform {
    float translate[3];
    float rotate[3];            /* degrees about x, y, z                                           */
    float scale[3];
    uint32_t flags;             /* RTC_XF_* bits                                                   */
} rtc_transform;

/* Axis-aligned box of six rectangles, centre and size (core/src/primitives/box.cuh, aarect.cuh).  Its
 * faces report the outward normal and front_face = true whatever side the ray comes from, as the
 * reference's xy/xz/yz_rect do; the faces at the low coordinate go through rt::flip_normals. */
typedef struct rtc_box {
    float center[3];
    float size[3];
    int32_t material;
    uint32_t transform;         /* 1-based index into rtc_scene_desc.transforms; 0 = none          */
} rtc_box;

/* Perspective camera (core/src/cameras/perspective_camera.cuh:41-117). */
typedef struct rtc_camera {
    float look_from[3];
    float look_at[3];
    float up[3];
    float vfov;        /* degrees                                                                  */
    float aspect;      /* the reference takes it from the CLI -ratio (scenes/scene_manager.cpp:83)  */
    float aperture;    /* lens_radius = aperture / 2                                               */
    float focus;       /* focus distance                                                           */
} rtc_camera;

typedef enum rtc_background_kind {
    RTC_BG_CONSTANT = 0,     /* camera::background_color (core/src/gpu.cu:741)                       */
    RTC_BG_SKY_GRADIENT = 1, /* lerp(bottom, top, 0.5*(unit.y+1)) of the ray direction               */
    RTC_BG_ENV_MAP = 2       /* equirectangular FP32 RGB map, lookup convention of get_spherical_uv
                                (core/src/utilities/uvmapping.cuh:144-158)                           */
} rtc_background_kind;

typedef struct rtc_background {
    int32_t kind;
    float color[3];          /* CONSTANT: the colour; SKY_GRADIENT: the colour at unit.y = -1      */
    float top[3];            /* SKY_GRADIENT: the colour at unit.y = +1                             */
    const float* env_rgb;    /* ENV_MAP: env_width*env_height*3 floats, top row first               */
    int32_t env_width;
    int32_t env_height;
} rtc_background;

typedef struct rtc_scene_desc {
    const rtc_texture* textures;      uint32_t num_textures;
    const rtc_image* images;          uint32_t num_images;
    const rtc_material* materials;    uint32_t num_materials;
    const rtc_dir_light* dir_lights;  uint32_t num_dir_lights;
    const rtc_sphere* spheres;        uint32_t num_spheres;
    const rtc_quad* quads;            uint32_t num_quads;
    const rtc_mesh* meshes;           uint32_t num_meshes;
    rtc_camera camera;
    rtc_background background;
    /* Further lights.  The light list holds omni lights, then directional lights, then spot lights, as
     * load_scene adds them (gpu.cu:504-523); that order also numbers them before the spheres. */
    const rtc_omni_light* omni_lights;  uint32_t num_omni_lights;
    const rtc_spot_light* spot_lights;  uint32_t num_spot_lights;
    /* Transforms and boxes.  *_transforms give, per sphere / quad / mesh, a 1-based index into
     * `transforms` (0 = none); each may be NULL when no object of that kind is transformed.  Boxes follow
     * the quads in the object order, as load_scene adds them (gpu.cu:527-565). */
    const rtc_transform* transforms;    uint32_t num_transforms;
    const uint32_t* sphere_transforms;
    const uint32_t* quad_transforms;
    const uint32_t* mesh_transforms;
    const rtc_box* boxes;               uint32_t num_boxes;
} rtc_scene_desc;

/* Triangle geometry read from a Wavefront OBJ file, laid out for rtc_mesh: per-vertex positions (and
 * normals / texture coordinates when the file has them, else NULL), 32-bit triangle indices.  Replaces
 * the reference's tinyobjloader path (core/src/utilities/mesh_loader.cuh), which keeps shape 0 only
 * (core/src/gpu.cu:628): here every object and group is merged, polygons are fan-triangulated and
 * negative (relative) indices are resolved.  Free with rtc_free_obj. */
typedef struct rtc_obj_mesh {
    float* vertices;          /* num_vertices*3                                                    */
    float* normals;           /* num_vertices*3 or NULL                                            */
    float* uvs;               /* num_vertices*2 or NULL                                            */
    uint32_t* indices;        /* num_triangles*3                                                   */
    uint32_t num_vertices;
    uint32_t num_triangles;
} rtc_obj_mesh;
rtc_status rtc_load_obj(const char* path, rtc_obj_mesh* mesh);
void rtc_free_obj(rtc_obj_mesh* mesh);

/* The reference's `.scene` files (libconfig syntax), read the way core/src/scenes/scene_loader.cpp reads
 * them into a sceneConfig and converted as rtc_sceneconfig.hpp converts one: image, camera, lights
 * (directional, omni, spot), solid / checker / image textures, lambertian / metal / glass materials,
 * spheres, quads and OBJ meshes (read with rtc_load_obj).  Values follow libconfig's typing as the
 * reference reads it (no AutoConvert): a float setting written as an integer (`radius = 1;`) keeps the
 * loader's default, and colours of three integers are 0-255 values.  Where scene_loader throws (a setting
 * handed to the builder with the wrong type, a nameless texture or material, a primitive without a
 * material) loading fails with RTC_ERR_BAD_SCENE, as does a syntax error (the message names the line).
 * Relative paths resolve against the scene file's directory, then the working directory.  What the
 * render path does not cover (other primitives, materials and textures, transforms, groups) is listed by
 * rtc_scene_file_skipped.  Replaces scene_loader::loadSceneFromFile (scene_loader.cpp:19-120) followed
 * by the scene_builder getters a caller of launchGPU passes on. */
typedef struct rtc_scene_file rtc_scene_file;
/* Image decoder for image textures: returns malloc'ed RGB8 pixels (width*height*3, top row first) that
 * the scene file frees with free(), or NULL.  Without one, image textures are skipped. */
typedef uint8_t* (*rtc_image_loader)(const char* path, int* width, int* height, void* user);
/* The reference's table capacities.  scene_loader counts each list into a uint8_t (scene_loader.cpp:
 * 124-204, 220-229, 280-282), so a kind holds (list length mod 256) entries, and it sizes the dielectric
 * table from a `dielectric` key while filling it from `glass` (scene_loader.cpp:191, 1092), so glass
 * materials, and the objects using them, are dropped unless a `dielectric` list makes room.  By default
 * every entry is kept; this flag reproduces the reference. */
#define RTC_SCENE_FILE_REFERENCE_CAPACITY 1
/* The reference's OBJ meshes.  load_scene renders the first meshes entry's file (meshes[0]) for every
 * entry (gpu.cu:626-631), each with its own material, and createObjMesh drops the entry's position and
 * transform (scene_factory.cuh:373-385).  By default each entry renders its own file, offset by its
 * position and transformed; this flag reproduces the reference. */
#define RTC_SCENE_FILE_REFERENCE_MESHES 2
typedef struct rtc_scene_file_info {
    int32_t width, height;     /* image.width / image.height (scene_builder's 400 x 225 when absent)  */
    int32_t spp, max_depth;    /* image.samplesPerPixel / image.maxDepth (50 / 100 when absent)      */
    uint32_t num_skipped;      /* notes readable with rtc_scene_file_skipped                          */
} rtc_scene_file_info;
rtc_status rtc_scene_file_load(const char* path, uint32_t flags, rtc_image_loader load_image, void* user,
                               rtc_scene_file** out);
/* The scene description (valid until rtc_scene_file_free), ready for rtc_scene_create. */
const rtc_scene_desc* rtc_scene_file_desc(const rtc_scene_file* file);
rtc_status rtc_scene_file_get_info(const rtc_scene_file* file, rtc_scene_file_info* info);
const char* rtc_scene_file_skipped(const rtc_scene_file* file, uint32_t index);
void rtc_scene_file_free(rtc_scene_file* file);

/* ------------------------------------------------------------------------------------------------ */
/* render parameters                                                                                 */
/* ------------------------------------------------------------------------------------------------ */

typedef enum rtc_mode {
    /* Reference semantics: one thrust::minstd_rand stream per pixel seeded seed + j*width + i and
     * consumed by all samples in order (core/src/gpu.cu:761-790), the 50/50 light/cosine mixture
     * for lambertian (camera.cuh:204-213), floor(sqrt(spp))^2 traced samples divided by spp
     * (gpu.cu:1989, color.cuh:289-300), and the other quirks of the reference's render path. */
    RTC_MODE_COMPAT = 0,
    /* Counter-based stream per (pixel, sample); samples of one pixel are independent, light-list
     * sampling only when the list is non-empty, cosine sampling otherwise, spp samples traced. */
    RTC_MODE_CLEAN = 1
} rtc_mode;

/* Order in which the reference's multi-draw expressions consume the stream.  The reference calls
 * get_real() several times inside one constructor call or one overloaded-operator expression
 * (random_in_unit_disk, random_in_unit_sphere: gpu_randomizer.cuh:61-76; directional_light::random:
 * directional_light.cuh:165-171), whose operand order C++ leaves unspecified.  g++ evaluates them
 * right to left; the CUDA front end left to right. */
typedef enum rtc_draw_order {
    RTC_DRAW_ORDER_DEVICE = 0,  /* as the reference's nvcc build consumes it (left to right)      */
    RTC_DRAW_ORDER_HOST = 1     /* as a g++ build of the reference's headers consumes it          */
} rtc_draw_order;

/* Execution engine.  Both compute bit-identical radiance for the same mode and draw order. */
typedef enum rtc_engine {
    RTC_ENGINE_AUTO = 0,        /* the library's choice (wavefront)                                       */
    RTC_ENGINE_MEGAKERNEL = 1,  /* one thread per pixel runs whole paths (the reference's kernel shape)   */
    RTC_ENGINE_WAVEFRONT = 2    /* extend / shade kernels over compacted path queues                      */
} rtc_engine;

typedef struct rtc_render_params {
    int32_t width;
    int32_t height;
    int32_t spp;
    int32_t max_depth;
    uint32_t seed;         /* reference: 2580 (core/src/gpu.cu:2080)                                 */
    int32_t mode;          /* rtc_mode                                                               */
    int32_t draw_order;    /* rtc_draw_order (COMPAT only)                                           */
    int32_t block_size;    /* 0 = library default                                                    */
    int32_t engine;        /* rtc_engine                                                             */
    int32_t flags;         /* RTC_FLAG_* bits                                                        */
} rtc_render_params;

/* Record CUDA events around every extend and shade launch of the wavefront engine; the per-kernel
 * device times are then reported by rtc_get_render_stats (extend_ms / shade_ms / *_launches). */
#define RTC_FLAG_KERNEL_TIMING 1
/* Traverse the 8-wide BVH with quantised child boxes (96-byte nodes: an 8-bit grid per axis, bounds
 * rounded outwards so no hit is lost) instead of the binary one (64-byte nodes, the default).  Both
 * hold the same leaves in the same order; the closest hit is the same except for which of several
 * primitives at exactly the same distance is reported.  A node-layout option for the batch autotuner;
 * scenes whose 8-wide tree would be too deep for its stack, and device-built trees, use the binary
 * nodes. */
#define RTC_FLAG_WIDE_BVH 2
/* Clean mode: split each pixel's samples into min(8, spp) consecutive groups that run on separate path
 * slots, so a pixel's samples trace in parallel instead of one after another (shorter critical path,
 * lower latency for an image).  Each group sums its samples in order, then the group sums are added in
 * group order: results are deterministic and the same in both engines, but differ from the one-group
 * sum in the last bits (float addition is not associative).  Needs per-image scratch: not available to
 * rtc_render_noalloc.  Compat mode ignores it (a pixel's samples share one stream there). */
#define RTC_FLAG_SAMPLE_GROUPS 4
/* Clean mode with an environment-map background: lambertian bounces also sample the map in proportion
 * to its luminance (x sin(theta)), with probability 0.2, mixed with their light and cosine sampling
 * (the mixture_pdf(objects, background_pdf, 0.8) that camera.cuh:333-336 leaves commented out, with
 * image_pdf's marginal and conditional CDFs, pdf/image_pdf.cuh:80-145).  The estimate stays unbiased
 * (the cosine part covers the hemisphere) and converges to the same image with less noise where the
 * map carries the light.  Compat mode ignores it (the reference's GPU path never samples its map,
 * gpu.cu:729-742). */
#define RTC_FLAG_ENV_SAMPLING 8

/* ------------------------------------------------------------------------------------------------ */
/* context and scenes                                                                                */
/* ------------------------------------------------------------------------------------------------ */

typedef struct rtc_context rtc_context;
typedef struct rtc_scene rtc_scene;

/* Creates a context on CUDA device `device` (the reference picks the first device, gpu.cu:92-116). */
rtc_status rtc_context_create(int device, rtc_context** out);
rtc_status rtc_context_destroy(rtc_context* ctx);

/* Flattens the description, builds the SAH BVH on the host and uploads everything to the device.
 * Replaces the reference's prepare* deep copies and its single-thread load_scene<<<1,1>>> build
 * (core/src/gpu.cu:862-1725, 481-751).  The description may be freed after the call. */
rtc_status rtc_scene_create(rtc_context* ctx, const rtc_scene_desc* desc, rtc_scene** out);
rtc_status rtc_scene_destroy(rtc_scene* scene);

/* BVH builders.  The reference builds its tree on one device thread (random axis, exchange sort of the
 * span, bvh_node.cuh:63-108 via gpu.cu:749); it has no choice of builder, so rtc_scene_create_ex and
 * the option below have no reference counterpart. */
#define RTC_BVH_SAH 0      /* binned SAH on host threads, leaves of up to 4 items, 8-wide copy (default) */
#define RTC_BVH_DEVICE 1   /* built on the device: primitives sorted by the 30-bit Morton code of their
                              centroids, then clustered bottom-up (PLOC: mutual nearest neighbours by
                              union surface area within 16 positions); one primitive per leaf, tree
                              quality close to SAH.  No 8-wide copy (RTC_FLAG_WIDE_BVH renders use the
                              binary nodes).  Falls back to RTC_BVH_SAH for a single primitive or a tree
                              deeper than the traversal stack. */
#define RTC_BVH_DEVICE_LBVH 2   /* built on the device as a linear BVH over the same sorted codes
                                   (Karras 2012): the fastest build, more node visits per ray.  Same
                                   limits and fallback as RTC_BVH_DEVICE. */
typedef struct rtc_scene_options {
    uint32_t bvh_builder;      /* RTC_BVH_*                                                          */
    uint32_t reserved[3];      /* zero                                                               */
} rtc_scene_options;
/* rtc_scene_create with options (NULL options: rtc_scene_create). */
rtc_status rtc_scene_create_ex(rtc_context* ctx, const rtc_scene_desc* desc, const rtc_scene_options* options,
                               rtc_scene** out);

typedef struct rtc_scene_info {
    uint32_t num_primitives;   /* lights + spheres + quads + triangles                             */
    uint32_t num_lights;
    uint32_t num_nodes;        /* BVH2 nodes                                                        */
    uint32_t max_leaf_size;
    uint64_t device_bytes;     /* bytes resident on the device for this scene                      */
    double build_ms;           /* validation, flattening and BVH build time (host wall clock)        */
    uint32_t bvh_builder;      /* RTC_BVH_* that built the tree                                      */
    uint32_t num_wide_nodes;   /* 8-wide nodes (RTC_FLAG_WIDE_BVH); 0: the scene has only binary nodes */
} rtc_scene_info;
rtc_status rtc_scene_get_info(const rtc_scene* scene, rtc_scene_info* info);

/* ------------------------------------------------------------------------------------------------ */
/* render                                                                                            */
/* ------------------------------------------------------------------------------------------------ */

/* Renders one image end to end with HOST output buffers (either may be NULL):
 *   radiance_sum: width*height*4 floats, the reference's per-pixel `pixel_color` sum over the traced
 *                 samples before prepare_pixel_color (RGB + alpha), frame-buffer order;
 *   rgb8:         width*height*3 bytes, int(255.99*clamp(sqrt(nan0(sum)/spp), 0, 0.999)) per channel,
 *                 PNG order (gpu.cu:792-799, 2098-2107).
 * Synchronous on the context's stream. */
rtc_status rtc_render(rtc_context* ctx, const rtc_scene* scene, const rtc_render_params* params,
                      float* radiance_sum, uint8_t* rgb8);

/* Same render with DEVICE output buffers (inputs already resident), on `stream`
 * (a cudaStream_t, or NULL for the context's stream).  d_radiance_sum must hold width*height
 * float4; d_rgb8 may be NULL.  d_counters, when not NULL, must hold 8 uint64 (zeroed by the caller)
 * and receives: rays traced (closest-hit traversals), paths traced, BVH nodes visited, primitive
 * tests, then the wavefront extend kernel's own rays, node visits and primitive tests, one unused.  The megakernel engine
 * returns without waiting for the GPU; the wavefront engine polls its queue counter between batches
 * of iterations and returns once the frame is complete. */
rtc_status rtc_render_device(rtc_context* ctx, const rtc_scene* scene, const rtc_render_params* params,
                             float* d_radiance_sum, uint8_t* d_rgb8, unsigned long long* d_counters,
                             void* stream);

/* Statistics of the last render on this context (wavefront engine): iterations of (extend, shade),
 * kernel launches, whether the drain kernel ran and for how many slots, and the device time of the
 * bulk iterations and of the drain kernel (ms, from CUDA events; the call waits for the render). */
typedef struct rtc_render_stats {
    uint32_t iterations;
    uint32_t launches;
    uint32_t drained_slots;
    uint32_t engine;
    float bulk_ms;
    float drain_ms;
    float extend_ms;           /* with RTC_FLAG_KERNEL_TIMING: summed device time of the extend launches */
    float shade_ms;            /* ... of the shade launches                                              */
    uint32_t extend_launches;
    uint32_t shade_launches;
} rtc_render_stats;
rtc_status rtc_get_render_stats(rtc_context* ctx, rtc_render_stats* stats);

/* Allocation-free render.  No counterpart in the reference: an addition for callers that cannot
 * allocate device memory when they render - code living under a memory budget fixed at start-up, a
 * process whose device allocator belongs to another framework, or a render issued where a cudaMalloc
 * would synchronise the device.  It runs the same wavefront kernels as rtc_render_device (same
 * results), with their path state in a 64 MiB static device array that every GPU loading this
 * library holds until exit, so it renders at most RTC_NOALLOC_MAX_PIXELS pixels per call (one path
 * slot per pixel) and rejects larger images with RTC_ERR_INVALID_ARGUMENT.  It allocates nothing
 * and needs no context: the scene (already on its device) and the 16-byte aligned device output
 * (width*height float4, frame-buffer order) come from the caller; `stream` may be NULL (legacy
 * stream).  The first call on a device looks up the array's address; make it before any stream
 * capture.  All calls share the array, so calls that overlap on the GPU race.  Returns when the frame
 * is complete; a call that fails part-way first waits for its queued kernels.  It always runs the
 * wavefront engine untimed (params->engine and RTC_FLAG_KERNEL_TIMING are ignored), and the calling
 * thread's current device is unchanged on return. */
#define RTC_NOALLOC_MAX_PIXELS 508376u
rtc_status rtc_render_noalloc(const rtc_scene* scene, const rtc_render_params* params, float* d_radiance_sum,
                              void* stream);

/* ------------------------------------------------------------------------------------------------ */
/* batched render                                                                                    */
/* ------------------------------------------------------------------------------------------------ */

/* One image of a batch.  The reference renders one image per launchGPU call (core/src/gpu.cu:2127);
 * a batch renders many images - different scenes, cameras, resolutions, spp and depths - through one
 * set of wavefront path slots and one extend/shade launch per iteration for all of them.  Each image
 * is computed exactly as rtc_render_device computes it alone (same per-pixel stream and sample order),
 * so its result does not depend on the rest of the batch. */
typedef struct rtc_job {
    const rtc_scene* scene;       /* resident scene (same device as the context)                         */
    const rtc_camera* camera;     /* NULL: the scene's own camera; else this job's camera                */
    rtc_render_params params;     /* width, height, spp, max_depth, seed of this image; mode and
                                     draw_order must be equal across the batch; engine, block_size and
                                     flags are ignored                                                   */
    float* d_radiance_sum;        /* device, width*height float4, 16-byte aligned, frame-buffer order    */
} rtc_job;

typedef struct rtc_batch_params {
    uint32_t slots;    /* path slots (pixels in flight); 0: min(total work units, 2^22), with 2^20 in
                          place of 2^22 when the first job is clean mode with RTC_FLAG_SAMPLE_GROUPS    */
    uint32_t ring;     /* job ring capacity, a power of two <= 65536; 0: 1024.  Larger batches are
                          admitted as earlier images complete.                                            */
    int32_t batch;     /* (extend, shade) iterations between two host polls; 0: 12.  A multiple of 6 is
                          replayed as a captured CUDA graph of six iterations                             */
    uint32_t drain;    /* queued slots below which the drain kernel finishes the batch; 0: 512 per SM;
                          1: no drain (every bounce runs in the extend/shade kernels)                     */
    unsigned long long* d_counters;   /* NULL, or 8 device uint64 (zeroed by the caller) that receive the
                          counts of rtc_render_device: rays, paths, node visits, primitive tests, then the
                          extend kernel's own rays, node visits and primitive tests                      */
    uint32_t block;    /* threads per block of the extend and shade kernels: 128, 256 or 512; 0: 128.
                          The grid keeps 1,024 threads per SM.                                            */
} rtc_batch_params;

/* Renders `num_jobs` images on `stream` (a cudaStream_t, or NULL for the context's stream) and returns
 * once all of them are complete.  `bp` may be NULL (defaults).  rtc_get_render_stats then reports the
 * batch's iterations, launches and drained slots. */
rtc_status rtc_render_batch(rtc_context* ctx, const rtc_job* jobs, uint32_t num_jobs, const rtc_batch_params* bp,
                            void* stream);

/* ------------------------------------------------------------------------------------------------ */
/* served render                                                                                     */
/* ------------------------------------------------------------------------------------------------ */

/* A render server on one device.  No counterpart in the reference, which renders one image per process
 * call (core/src/gpu.cu:2127).  Requests (scene, camera, resolution, spp, depth) are submitted from any
 * thread while others are on the GPU; a server thread admits them into the running job-ring wavefront
 * as ring entries and device memory free up (continuous batching), and copies each result to the
 * caller's host buffer when its last pixel is written.  Scenes are registered once (host BVH build) and
 * kept resident on the device under an HBM budget: a request whose scene is not resident uploads it,
 * evicting the least recently used scenes that no request in flight uses.  Each request is computed
 * exactly as rtc_render_device computes that image alone. */
typedef struct rtc_server rtc_server;

typedef struct rtc_server_config {
    int32_t device;
    int32_t mode;                /* rtc_mode, shared by every request                                  */
    int32_t draw_order;          /* rtc_draw_order (COMPAT), shared by every request                   */
    int32_t batch;               /* (extend, shade) iterations between two host polls; 0: 12           */
    uint32_t slots;              /* path slots; 0: 2^20 (fewer slots in flight: shorter iterations,     
                                    lower latency)                                                      */
    uint32_t ring;               /* requests in flight at most (power of two <= 65536); 0: 1024        */
    uint64_t hbm_budget_bytes;   /* device bytes for slots, resident scenes and request outputs;
                                    0: 120 GB                                                           */
    int32_t flags;               /* RTC_FLAG_* applied to every request (e.g. RTC_FLAG_SAMPLE_GROUPS)    */
    uint32_t bvh_builder;        /* RTC_BVH_* for rtc_server_add_scene                                  */
} rtc_server_config;

typedef struct rtc_request {
    uint32_t scene_id;           /* from rtc_server_add_scene                                          */
    int32_t use_scene_camera;    /* nonzero: the scene's own camera; zero: `camera`                     */
    rtc_camera camera;
    int32_t width, height, spp, max_depth;
    uint32_t seed;
} rtc_request;

typedef enum rtc_request_state {
    RTC_REQ_QUEUED = 0,          /* waiting for a ring entry or device memory                           */
    RTC_REQ_RUNNING = 1,         /* admitted, pixels in flight                                          */
    RTC_REQ_COPYING = 2,         /* complete on the device, result on its way to the host buffer        */
    RTC_REQ_DONE = 3,
    RTC_REQ_FAILED = 4
} rtc_request_state;

typedef struct rtc_request_info {
    int32_t state;               /* rtc_request_state                                                   */
    int32_t scene_uploaded;      /* 1 when admitting this request uploaded its scene (cache miss)       */
    double submit_ms;            /* server clock: ms since rtc_server_create                            */
    double admit_ms;
    double done_ms;              /* result in the caller's buffer                                       */
    uint64_t paths;              /* traced camera samples of the image                                  */
} rtc_request_info;

typedef struct rtc_server_stats {
    uint64_t submitted, completed, failed;
    uint64_t paths;                       /* traced camera samples of completed requests                */
    uint64_t scene_uploads, scene_evictions;
    uint64_t resident_bytes, peak_resident_bytes;   /* slots + resident scenes + request outputs       */
    uint64_t iterations, launches;
    uint32_t queued, in_flight;
} rtc_server_stats;

rtc_status rtc_server_create(const rtc_server_config* cfg, rtc_server** out);
/* Stops the server: queued requests fail, requests in flight complete first. */
rtc_status rtc_server_destroy(rtc_server* server);
/* Registers a scene: validation, flattening and BVH build on the host (rtc_scene_create's work).  The
 * description may be freed after the call; the scene uploads on its first request. */
rtc_status rtc_server_add_scene(rtc_server* server, const rtc_scene_desc* desc, uint32_t* scene_id);
/* Queues a request.  `radiance_sum` (host, width*height*4 floats, frame-buffer order, as rtc_render
 * writes it; any host memory) receives the result and must stay valid until the request is done.  The
 * device-to-host copy goes through page-locked staging buffers the server keeps for reuse. */
rtc_status rtc_server_submit(rtc_server* server, const rtc_request* req, float* radiance_sum, uint64_t* ticket);
/* RTC_OK once the request is done (its record is released), RTC_ERR_BUSY while queued, running or
 * copying, RTC_ERR_NOT_FOUND for an unknown ticket; `info` (may be NULL) is filled in every case. */
rtc_status rtc_server_poll(rtc_server* server, uint64_t ticket, rtc_request_info* info);
/* Blocks until the request is done (RTC_OK, record released) or `timeout_ms` passes (RTC_ERR_TIMEOUT;
 * a negative timeout waits without limit).  A failed request returns its error. */
rtc_status rtc_server_wait(rtc_server* server, uint64_t ticket, int32_t timeout_ms, rtc_request_info* info);
rtc_status rtc_server_get_stats(rtc_server* server, rtc_server_stats* stats);

/* Closest-hit queries on arbitrary rays (hit-identity tests).  rays: n x 8 floats
 * (ox, oy, oz, tmin, dx, dy, dz, tmax) in host memory; `depth`/`max_depth` decide light visibility as
 * in the reference's world.hit (directional_light.cuh:106).  Outputs (host, n each, may be NULL):
 * prim_id (-1 on a miss) and t. */
rtc_status rtc_trace_closest(rtc_context* ctx, const rtc_scene* scene, const float* rays, uint32_t n,
                             int32_t depth, int32_t max_depth, int32_t* prim_id, float* t);
/* rtc_trace_closest with render flags: RTC_FLAG_WIDE_BVH walks the 8-wide nodes (where the scene has
 * them), so both node layouts can be checked against each other.  No counterpart in the reference. */
rtc_status rtc_trace_closest_ex(rtc_context* ctx, const rtc_scene* scene, const float* rays, uint32_t n,
                                int32_t depth, int32_t max_depth, int32_t flags, int32_t* prim_id, float* t);

/* ------------------------------------------------------------------------------------------------ */
/* drop-in form of the reference call                                                                */
/* ------------------------------------------------------------------------------------------------ */

/* launchGPU (core/src/gpu.cu:2127) with the reference's semantics: compat mode, seed 2580, one image,
 * 8-bit PNG written to `filepath` (rows flipped).  tx/ty are accepted for signature compatibility
 * (the reference's block shape, gpu.cu:2072-2080) and otherwise ignored.  Unlike the reference it
 * returns a status instead of exiting, and prints nothing unless quiet_mode is 0. */
rtc_status rtc_launchGPU(const rtc_scene_desc* scene, int width, int height, int spp, int max_depth,
                         int tx, int ty, const char* filepath, int quiet_mode);

/* Writes an 8-bit RGB PNG (top row first). */
rtc_status rtc_write_png(const char* filepath, const uint8_t* rgb8, int width, int height);

#ifdef __cplusplus
}
#endif

#endif /* RTC_H */
