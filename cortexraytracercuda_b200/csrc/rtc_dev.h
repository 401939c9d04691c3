// rtc_dev.h - device-resident scene layout (shared by the host builder and the kernels).
//
// HBM layout, all arrays 16-byte aligned float4/int4 so every fetch is one vectorised load:
//
//   nodes      BVH2, 4 x float4 = 64 B per node:
//                n0 = (L.lo.x, L.hi.x, L.lo.y, L.hi.y)   n1 = (R.lo.x, R.hi.x, R.lo.y, R.hi.y)
//                n2 = (L.lo.z, L.hi.z, R.lo.z, R.hi.z)   n3 = (child L, child R, -, -) as int bits
//              child >= 0: inner node index; child < 0: leaf, ~child = (first_item << 5) | count.
//   nodes8     the same tree collapsed to 8-wide nodes with quantised child boxes, 5 x float4 = 80 B:
//                (p.xyz, header)  header = (e.x+127) | (e.y+127) << 8 | (e.z+127) << 16 | valid << 24
//                (child base, item base, link bytes of slots 0-3, link bytes of slots 4-7) as int bits
//                (qlo.x[0..7] bytes, qhi.x[0..7] bytes) (same for y) (same for z)
//              slot s's box on axis a is [p.a + qlo.a[s] * 2^e.a, p.a + qhi.a[s] * 2^e.a] (rounded outwards
//              when built, so it encloses the child's exact box); `valid` has a bit per slot in use.
//              Bit k of s is the high side of axis k (children placed by the direction of their centre
//              from the node's).  Link byte: 0x80 | r for an inner child, node = child base + r (a node's
//              inner children are consecutive); (count - 1) << 5 | offset for a leaf, whose items are
//              items8[item base + offset ...] (count 1-4).  Renders use it when RTC_FLAG_WIDE_BVH is set.
//   items8     uint32 per 8-wide leaf entry: the same item words as `items`, regrouped so that the leaves
//              of one wide node are consecutive.
//   items      uint32 per leaf entry, leaf order: (kind << 29) | index into that kind's array.
//   xprim      int4 per transformed primitive or box face (leaf order): (transform or -1, inner kind,
//              inner index, global id).  The inner record sits in the sph / quad / tri / rect array.
//              Xprims have their own BVH2 (`xnodes`, leaves into `xitems`), walked after the main one.
//   xf         8 x float4 per transform: (translate.xyz, flags) (scale.xyz, -) (inverse rotation columns
//              0..2, xyz) (forward rotation columns 0..2, xyz), the glm matrices of rt::rotate
//   rect       2 x float4 per box face: (a0, a1, b0, b1) (k, axis, flip, material); axis 0 = xy_rect
//              (plane z = k), 1 = xz_rect (y = k), 2 = yz_rect (x = k)
//   sph        float4 (center.xyz, radius)                      16 B / sphere  (leaf order)
//   sph_aux    int2   (material, global id)
//   tri        3 x float4: (v0.xyz, material bits) (v1-v0, gid bits) (v2-v0, smooth-normal slot or -1)
//                                                               48 B / triangle test (leaf order)
//   tri_n      float4 (middle_normal.xyz, -)                    fetched once per final hit only
//   tri_vn     3 x float4 vertex normals (unit_vector'd) for smooth triangles
//   tri_uv     2 x float4 per triangle, only when a mesh has texture coordinates: (uv0.xy, uv1.xy) (uv2.xy, -)
//   quad       5 x float4: (n.xyz, D) (Q.xyz, mat) (u.xyz, gid) (v.xyz, -) (w.xyz, -)
//   light      6 x float4 per light, in light-list order (omni, directional, spot lights):
//              directional (quad): (n.xyz, D) (P.xyz, mat) (u.xyz, gid) (v.xyz, invisible) (w.xyz, area)
//                                  (emit.rgb, intensity)
//              omni / spot (sphere): (center.xyz, radius) (-, -, -, mat) (spot direction.xyz, gid)
//                                  (cos cutoff, falloff, -, invisible) (-, -, -, -1: the sphere marker)
//                                  (emit.rgb, intensity)
//   materials  int4 (kind, texture, -, -) + float4 (fuzz, ior, intensity, directional)
//   textures   int4 (kind, even, odd, image) + float4 (color.rgb, inv_scale)
//   images     int4 (byte offset, width, height, -) into image_bytes
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Kernels that walk the xprim BVH (transformed primitives and box faces) are compiled separately, with
// RTC_XP=1, into the inline namespace rtc::xp1; without them the traversal carries none of that code.
#ifndef RTC_XP
#define RTC_XP 0
#endif
#if RTC_XP
#define RTC_XP_NS xp1
#else
#define RTC_XP_NS xp0
#endif

namespace rtc {

enum ItemKind : uint32_t { ITEM_SPHERE = 0, ITEM_QUAD = 1, ITEM_TRI = 2, ITEM_LIGHT = 3, ITEM_XPRIM = 4 };
// Item word: (kind << ITEM_KIND_SHIFT) | index into that kind's array.
constexpr uint32_t ITEM_KIND_SHIFT = 29;
constexpr uint32_t ITEM_INDEX_MASK = (1u << ITEM_KIND_SHIFT) - 1u;
// Inner kinds of an xprim: ITEM_SPHERE, ITEM_QUAD, ITEM_TRI, or a box face.
constexpr int XPRIM_RECT = 5;
// Material kinds past the public rtc_material_kind values: a spot light's diffuse_spot_light.
constexpr int MAT_SPOT_LIGHT = 4;
constexpr int LEAF_COUNT_BITS = 5;
constexpr int MAX_LEAF = 31;
constexpr int TRAVERSAL_STACK = 64;
constexpr int TRAVERSAL_STACK8 = 64;   // 8-wide: one pending group (node, slots left) per level
constexpr int NODE8_FLOATS = 20;       // 5 x float4 per 8-wide node

// kernel status word bits (device -> host)
enum StatusBits : uint32_t {
    STATUS_STACK_OVERFLOW = 1u,
    STATUS_BAD_ITEM = 2u,
    STATUS_BAD_MATERIAL = 4u,
    STATUS_BAD_TEXTURE = 8u,
    STATUS_TIMEOUT = 16u,
};

struct DevCamera {
    float origin[3];
    float llc[3];
    float horizontal[3];
    float vertical[3];
    float u[3];
    float v[3];
    float lens_radius;
    float time0, time1;
};

struct DevBackground {
    int kind;
    float color[3];
    float top[3];
    const float* env;   // device, env_w*env_h*3
    int env_w, env_h;
    // environment-map importance sampling (clean mode, RTC_FLAG_ENV_SAMPLING; null otherwise): the
    // marginal CDF over rows (env_h floats, top row first) followed by each row's conditional CDF over
    // its columns (env_w floats per row), of luminance x sin(theta); pdf_scale = W*H / (2 pi^2)
    const float* cdf;
    float pdf_scale;
};

struct DevScene {
    const float4* nodes;
    const float4* nodes8;      // null: binary traversal
    const uint32_t* items;
    const uint32_t* items8;    // the 8-wide nodes' leaf items (with nodes8)
    const float4* sph;
    const int2* sph_aux;
    const float4* tri;
    const float4* tri_n;
    const float4* tri_vn;
    const float4* tri_uv;      // null, or 2 x float4 per triangle: (uv0, uv1) (uv2, -) in leaf order
    const float4* quad;
    const float4* light;
    const int4* mat_i;
    const float4* mat_f;
    const int4* tex_i;
    const float4* tex_f;
    const int4* images;
    const uint8_t* image_bytes;
    const int4* xprim;
    const float4* xf;
    const float4* rect;
    const float4* xnodes;      // BVH2 over the xprims (null when there are none)
    const uint32_t* xitems;
    uint32_t num_nodes;
    uint32_t num_nodes8;
    uint32_t num_items;
    uint32_t num_lights;
    uint32_t num_materials;
    uint32_t num_textures;
    uint32_t num_images;
    uint32_t num_sph, num_tri, num_quad;
    uint32_t num_xprim, num_xf, num_rect, num_xnodes, num_xitems;
    DevCamera cam;
    DevBackground bg;
};

// Per-launch parameters.
struct DevParams {
    int width, height;
    int spp;           // as given (compat divides by it)
    int sqrt_spp;      // compat: int(sqrt(spp))
    int max_depth;
    uint32_t seed;
    int draw_order;    // 0 device (left to right), 1 host (right to left)
    int64_t num_pixels;
    int groups;        // sample groups per pixel (clean mode, RTC_FLAG_SAMPLE_GROUPS), else 1
    uint8_t* rgb8;     // non-null: each finished pixel is also written quantised here (quantize_pixel)
};

// Wavefront path slots (one slot = one pixel, or one sample group, in flight) and the slot queues.
//
// A slot's path state is one 96-byte record of three 32-byte sectors, each moved by a single 256-bit
// load or store (the kernels reach slots through the queues, so neighbouring lanes touch unrelated
// records: a sector per access is the least a scattered access can move):
//   sector 0, ray:    origin.xyz, direction.xyz, the trace's start (0 for an ordinary ray, t + 0.001 for
//                     the re-hit from behind a one-sided light, camera.cuh:177-183), and the depth word
//                     (depth left in the low 16 bits | job slot in the high 16 bits, 0 for one image);
//   sector 1, shade:  path attenuation rgb, radiance of the current sample rgb, and the closest hit the
//                     extend kernel found (t, item bits; 0xffffffff = miss);
//   sector 2, pixel:  pixel (0xffffffff = idle slot), sample index, the minstd state (compat) or the
//                     sample group (clean), the PCG32 state's low word (clean), the pixel sum rgb, and
//                     the PCG32 state's high word.  A clean-mode stream's increment is 2 s + 1 for sample
//                     s (Pcg32::seed), so it is recomputed from the sample index, not stored.
// The ray's time (perspective_camera::get_ray draws it) is not kept: no hit test reads it.
constexpr uint32_t WF_REC_WORDS = 24;
constexpr uint32_t WF_REC_BYTES = WF_REC_WORDS * 4;
struct WfBuffers {
    uint32_t* rec;        // slots x WF_REC_WORDS words, 256-byte aligned (so every sector is 32-byte aligned)
    uint32_t* queue[3];   // [0], [1]: the alternating slot queues; [2]: slots split off as long chains
    uint32_t* ctr;        // [0..2] queue sizes (rotating), [3] next pixel to fetch, [4] long-chain queue size
    uint32_t slots;
};

constexpr uint32_t WF_IDLE = 0xffffffffu;
constexpr int WF_MAX_DEPTH = 0xffff;
constexpr uint32_t WF_MAX_JOBS = 1u << 16;   // job ring capacity limit (job slot in 16 bits)
__host__ __device__ __forceinline__ uint32_t wf_depth(uint32_t w) { return w & 0xffffu; }
__host__ __device__ __forceinline__ uint32_t wf_job(uint32_t w) { return w >> 16; }
__host__ __device__ __forceinline__ uint32_t wf_pack(uint32_t depth, uint32_t job) { return (job << 16) | depth; }

// One image of a batched or served render: a record in the device job ring.
struct DevJob {
    DevScene S;                  // the scene's arrays, with this job's camera
    DevParams P;
    float4* out;                 // width*height radiance sums, frame-buffer order
    unsigned long long begin;    // first index of the job's work units (pixel x sample group) in the
                                 // engine's global sequence
    float4* part;                // P.groups > 1: width*height*groups partial sums
    uint32_t* gcnt;              // P.groups > 1: per pixel, groups finished (zero at admission)
};

// Hand-out state of the global pixel sequence (device).  Pixels [next, limit) are admitted and not yet
// claimed; jobs with sequence numbers in [lo, hi) may own them (ring slot = sequence & mask).
struct WfWindow {
    unsigned long long limit;
    uint32_t lo, hi;
};
struct WfFeed {
    unsigned long long next;
    WfWindow win;
    uint32_t pad[2];
};

// Kernel arguments of the two job sources (the device-side policy types in rtc_wavefront.cuh add
// their methods to these).
struct WfOneArgs {             // one image
    DevScene S;
    DevParams P;
    float4* out;
    float4* part;              // P.groups > 1: partial sums (width*height*groups)
    uint32_t* gcnt;            // P.groups > 1: per-pixel count of finished groups (zeroed per render)
};
struct WfTableArgs {           // a ring of jobs
    const DevJob* jobs;
    WfFeed* feed;
    uint32_t* done;            // per ring slot: pixels written
    uint32_t mask;             // ring capacity - 1 (a power of two)
};

// Iteration k reads queue (k & 1) with size ctr[k % 3], appends to queue ((k+1) & 1) counted in
// ctr[(k+1) % 3] and clears ctr[(k+2) % 3], which iteration k+1 appends to.
// [5], [6]: the next queue entry the extend / shade kernel hands out (each kernel clears the other's)
enum WfCtr { WF_NEXT_PIXEL = 3, WF_LONG = 4, WF_FETCH_EXTEND = 5, WF_FETCH_SHADE = 6, WF_CTR_N = 7 };
struct WfIter {
    int qin, cin, cout, czero;
};
inline __host__ __device__ WfIter wf_iter(uint64_t k) {
    WfIter w;
    w.qin = (int)(k & 1u);
    w.cin = (int)(k % 3u);
    w.cout = (int)((k + 1u) % 3u);
    w.czero = (int)((k + 2u) % 3u);
    return w;
}

// Counters (unsigned long long on device).
// Totals of the render, then the wavefront extend kernel's own share.
enum CounterIdx {
    CNT_RAYS = 0, CNT_PATHS = 1, CNT_NODES = 2, CNT_PRIMS = 3,
    CNT_EXT_RAYS = 4, CNT_EXT_NODES = 5, CNT_EXT_PRIMS = 6, CNT_N = 8
};

}  // namespace rtc
