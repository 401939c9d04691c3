// rtc_api.cpp - the C ABI (include/rtc.h): contexts, scene flattening + upload, render dispatch, PNG.
//
// Host float arithmetic that feeds the kernels (quad/light planes, triangle edges and normals, the
// camera frame) restates the reference's constructors operation by operation and is compiled with
// -ffp-contract=off, so the device sees bit-identical values to what a g++ build of the reference
// computes.
#include "../../include/rtc.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "bvh_build.h"
#include "rtc_dev.h"
#include "rtc_kernels.h"
#include "rtc_internal.h"
#include "rtc_objects.h"
#include "rtc_math.cuh"

using namespace rtc;

namespace {
thread_local std::string g_err;

rtc_status fail(rtc_status s, const std::string& msg) {
    g_err = msg;
    return s;
}
rtc_status cuda_fail(cudaError_t e, const char* what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? RTC_ERR_OOM : RTC_ERR_CUDA;
}
#define RTC_CUDA(call)                                   \
    do {                                                 \
        cudaError_t _e = (call);                         \
        if (_e != cudaSuccess) return cuda_fail(_e, #call); \
    } while (0)

bool finite3(const float* p) { return std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]); }

}  // namespace

extern "C" const char* rtc_last_error_string(void) { return g_err.c_str(); }

extern "C" rtc_status rtc_context_create(int device, rtc_context** out) {
    if (!out) return fail(RTC_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0) return fail(RTC_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= n) return fail(RTC_ERR_INVALID_ARGUMENT, "device index out of range");
    cudaDeviceProp prop;
    RTC_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(RTC_ERR_NO_DEVICE, std::string("device is not sm_100: ") + prop.name);
    RtcDeviceScope dev(device);
    RTC_CUDA(dev.error());
    rtc_context* c = new (std::nothrow) rtc_context();
    if (!c) return fail(RTC_ERR_OOM, "host allocation failed");
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    cudaError_t e1 = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    cudaError_t e2 = cudaMalloc(&c->d_status, sizeof(uint32_t));
    cudaError_t e3 = cudaMalloc(&c->d_counters, CNT_N * sizeof(unsigned long long));
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
        cudaError_t e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
        rtc_context_destroy(c);
        return cuda_fail(e, "context setup");
    }
    *out = c;
    return RTC_OK;
}

extern "C" rtc_status rtc_context_destroy(rtc_context* c) {
    if (!c) return RTC_OK;
    RtcDeviceScope dev(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->engine.reset();
    cudaFree(c->d_status);
    cudaFree(c->d_counters);
    cudaFree(c->d_out);
    cudaFree(c->d_rgb8);
    cudaFree(c->d_wf);
    cudaFree(c->d_groups);
    cudaFree(c->d_batch_groups);
    if (c->h_poll) cudaFreeHost(c->h_poll);
    for (cudaEvent_t& e : c->poll_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : c->phase_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : c->split_ev)
        if (e) cudaEventDestroy(e);
    if (c->stream_long) cudaStreamDestroy(c->stream_long);
    for (cudaEvent_t e : c->kev) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return RTC_OK;
}

// ---------------------------------------------------------------------------------------------------
// scene flattening
// ---------------------------------------------------------------------------------------------------
namespace {

struct PlanarPre {    // quad / directional light constants (quad.cuh:55-67, directional_light.cuh:45-58)
    V3 n, normal, w;
    float D, area;
};
PlanarPre planar_pre(V3 pos, V3 u, V3 v) {
    PlanarPre p;
    p.n = cross(u, v);
    p.normal = unit(p.n);
    p.D = dot(p.normal, pos);
    p.w = divs(p.n, dot(p.n, p.n));
    p.area = len(p.n);
    return p;
}

// Conservative padding so the FMA slab test never culls a primitive its exact test accepts.  The slab
// distance fma(lo, 1/d, -o/d) carries an absolute error of about 2^-24 |o| / |d| from the rounded o/d,
// so a flat box (an axis-aligned quad or triangle: zero extent on one axis) near the world origin seen
// from a far ray origin needs padding in proportion to the ray origin's magnitude, not to its own
// coordinates.  `scene_scale` bounds |o| for every secondary ray (the largest coordinate of any
// primitive) and for primary rays from the scene's camera; 2^-21 of it covers origins up to about
// four times farther out.
Aabb pad_box(Aabb b, float scene_scale) {
    for (int k = 0; k < 3; ++k) {
        float m = std::max(std::fabs(b.lo[k]), std::fabs(b.hi[k]));
        float e = 1e-5f * m + 1e-6f + 1e-5f * (b.hi[k] - b.lo[k]) + 0x1p-21f * scene_scale;
        b.lo[k] -= e;
        b.hi[k] += e;
    }
    return b;
}
// Unpadded bounds of n points (pad_box follows once the scene's scale is known).
Aabb box_of(const V3* pts, int n) {
    Aabb b;
    for (int k = 0; k < 3; ++k) { b.lo[k] = INFINITY; b.hi[k] = -INFINITY; }
    for (int i = 0; i < n; ++i) {
        const float c[3] = {pts[i].x, pts[i].y, pts[i].z};
        for (int k = 0; k < 3; ++k) { b.lo[k] = std::min(b.lo[k], c[k]); b.hi[k] = std::max(b.hi[k], c[k]); }
    }
    return b;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// glm::rotate(m, angle, axis) for a coordinate axis (glm/ext/matrix_transform.inl:18-46), in float and
// in the same operation order; the axis is a unit vector, which normalize leaves unchanged.  `m` is
// column-major (m[column][row]).
void glm_rotate_axis(float m[4][4], float angle, int ax) {
    const float c = std::cos(angle), s = std::sin(angle);
    float axis[3] = {0.0f, 0.0f, 0.0f};
    axis[ax] = 1.0f;
    const float temp[3] = {(1.0f - c) * axis[0], (1.0f - c) * axis[1], (1.0f - c) * axis[2]};
    float R[3][3];
    R[0][0] = c + temp[0] * axis[0];
    R[0][1] = temp[0] * axis[1] + s * axis[2];
    R[0][2] = temp[0] * axis[2] - s * axis[1];
    R[1][0] = temp[1] * axis[0] - s * axis[2];
    R[1][1] = c + temp[1] * axis[1];
    R[1][2] = temp[1] * axis[2] + s * axis[0];
    R[2][0] = temp[2] * axis[0] + s * axis[1];
    R[2][1] = temp[2] * axis[1] - s * axis[0];
    R[2][2] = c + temp[2] * axis[2];
    float out[3][4];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 4; ++i) out[j][i] = (m[0][i] * R[j][0] + m[1][i] * R[j][1]) + m[2][i] * R[j][2];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 4; ++i) m[j][i] = out[j][i];
}

// rt::rotate's matrix (rotate.cuh hit()): identity, then glm::rotate about x, y and z by
// degrees_to_radians(sign * angle) = sign * angle * M_PI / 180.0f with the reference's float M_PI.
void rotate_matrix(const float deg[3], float sign, float m[4][4]) {
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i) m[j][i] = i == j ? 1.0f : 0.0f;
    for (int ax = 0; ax < 3; ++ax) glm_rotate_axis(m, (sign * deg[ax]) * 3.14159265358979323846f / 180.0f, ax);
}

// Device transform record (rtc_dev.h `xf`): 8 float4.
void put_transform(const rtc_transform& T, std::vector<float4>& xf) {
    float inv[4][4], fwd[4][4];
    rotate_matrix(T.rotate, -1.0f, inv);
    rotate_matrix(T.rotate, 1.0f, fwd);
    xf.push_back(make_float4(T.translate[0], T.translate[1], T.translate[2], ibits((int32_t)(T.flags & 7u))));
    xf.push_back(make_float4(T.scale[0], T.scale[1], T.scale[2], 0.0f));
    for (int j = 0; j < 3; ++j) xf.push_back(make_float4(inv[j][0], inv[j][1], inv[j][2], 0.0f));
    for (int j = 0; j < 3; ++j) xf.push_back(make_float4(fwd[j][0], fwd[j][1], fwd[j][2], 0.0f));
}

// World-space bounds of an object-space box seen through transform T: the corners mapped by the exact
// inverse of the ray's path into object space (o -> o / s -> R_inv o -> o - t), i.e. x -> s * R_inv^T
// (x + t), in double, padded for the float rounding of that path.
Aabb transform_box(const rtc_transform& T, const Aabb& b) {
    float inv[4][4];
    rotate_matrix(T.rotate, -1.0f, inv);
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    double mag = 0.0;
    for (int c = 0; c < 8; ++c) {
        double p[3] = {(c & 1) ? b.hi[0] : b.lo[0], (c & 2) ? b.hi[1] : b.lo[1], (c & 4) ? b.hi[2] : b.lo[2]};
        if (T.flags & RTC_XF_TRANSLATE)
            for (int k = 0; k < 3; ++k) p[k] += T.translate[k];
        mag = std::max({mag, std::fabs(p[0]), std::fabs(p[1]), std::fabs(p[2])});
        if (T.flags & RTC_XF_ROTATE) {
            // R_inv^T p: row k of the transpose is column k of R_inv
            double q[3];
            for (int k = 0; k < 3; ++k) q[k] = inv[k][0] * p[0] + inv[k][1] * p[1] + inv[k][2] * p[2];
            for (int k = 0; k < 3; ++k) p[k] = q[k];
        }
        if (T.flags & RTC_XF_SCALE)
            for (int k = 0; k < 3; ++k) p[k] *= T.scale[k];
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    double smax = 1.0;
    if (T.flags & RTC_XF_SCALE) smax = std::max({std::fabs((double)T.scale[0]), std::fabs((double)T.scale[1]), std::fabs((double)T.scale[2])});
    const double e = 4e-6 * mag * smax + 1e-6;
    Aabb r;
    for (int k = 0; k < 3; ++k) { r.lo[k] = (float)(lo[k] - e); r.hi[k] = (float)(hi[k] + e); }
    return r;
}

}  // namespace

// perspective_camera::initialize (perspective_camera.cuh:41-108), operation by operation.
bool rtc_make_camera(const rtc_camera& C, DevCamera& cam) {
    cam = DevCamera{};
    float theta = C.vfov * 3.14159265358979323846f / 180.0f;   // degrees_to_radians (math_utils.cuh)
    float half_height = std::tan(theta / 2.0f);
    float ratio = C.aspect;
    float focus = C.focus;
    V3 lookfrom = v3(C.look_from), lookat = v3(C.look_at), vup = v3(C.up);
    V3 w = unit(sub(lookfrom, lookat));
    V3 u = unit(cross(vup, w));
    V3 v = cross(w, u);
    float half_width = ratio * half_height;
    V3 origin = lookfrom;
    V3 llc = sub(sub(sub(origin, mul(half_width * focus, u)), mul(half_height * focus, v)), mul(focus, w));
    V3 horizontal = mul(2.0f * half_width * focus, u);
    V3 vertical = mul(2.0f * half_height * focus, v);
    const V3 vals[6] = {origin, llc, horizontal, vertical, u, v};
    float* dst[6] = {cam.origin, cam.llc, cam.horizontal, cam.vertical, cam.u, cam.v};
    for (int k = 0; k < 6; ++k) { dst[k][0] = vals[k].x; dst[k][1] = vals[k].y; dst[k][2] = vals[k].z; }
    cam.lens_radius = C.aperture / 2.0f;
    cam.time0 = 0.0f;
    cam.time1 = 1.0f;
    return std::isfinite(cam.llc[0] + cam.llc[1] + cam.llc[2] + horizontal.x + vertical.y);
}

const DevScene& rtc_scene_dev(const rtc_scene* s) { return s->dev; }

DevScene rtc_scene_view(const rtc_scene* s, const rtc_render_params* p) {
    DevScene S = s->dev;
    if (!p || !(p->flags & RTC_FLAG_WIDE_BVH)) S.nodes8 = nullptr;
    rtc_view_env_sampling(S, p);
    return S;
}
void rtc_view_env_sampling(DevScene& S, const rtc_render_params* p) {
    if (!p || !(p->flags & RTC_FLAG_ENV_SAMPLING) || p->mode != RTC_MODE_CLEAN) S.bg.cdf = nullptr;
}
DevParams rtc_dev_params(const rtc_render_params* p);

rtc_status rtc_build_host_scene(const rtc_scene_desc* d, HostScene& H, uint32_t bvh_builder, int device) {
    if (!d) return fail(RTC_ERR_INVALID_ARGUMENT, "null argument");
    if (bvh_builder != RTC_BVH_SAH && bvh_builder != RTC_BVH_DEVICE && bvh_builder != RTC_BVH_DEVICE_LBVH)
        return fail(RTC_ERR_INVALID_ARGUMENT, "unknown BVH builder");
    auto t0 = std::chrono::steady_clock::now();
    // ---- validation --------------------------------------------------------------------------
    auto bad = [&](const std::string& m) { return fail(RTC_ERR_BAD_SCENE, m); };
    if ((d->num_textures && !d->textures) || (d->num_images && !d->images) || (d->num_materials && !d->materials) ||
        (d->num_dir_lights && !d->dir_lights) || (d->num_spheres && !d->spheres) || (d->num_quads && !d->quads) ||
        (d->num_omni_lights && !d->omni_lights) || (d->num_spot_lights && !d->spot_lights) ||
        (d->num_meshes && !d->meshes))
        return bad("count > 0 with a null array");
    for (uint32_t i = 0; i < d->num_images; ++i)
        if (!d->images[i].rgb || d->images[i].width <= 0 || d->images[i].height <= 0) return bad("bad image " + std::to_string(i));
    for (uint32_t i = 0; i < d->num_textures; ++i) {
        const rtc_texture& t = d->textures[i];
        if (t.kind == RTC_TEX_SOLID) continue;
        if (t.kind == RTC_TEX_CHECKER) {
            if (t.even < 0 || (uint32_t)t.even >= d->num_textures || t.odd < 0 || (uint32_t)t.odd >= d->num_textures)
                return bad("checker texture " + std::to_string(i) + " references a missing texture");
            if (!(t.scale != 0.0f) || !std::isfinite(t.scale)) return bad("checker texture with zero scale");
            continue;
        }
        if (t.kind == RTC_TEX_IMAGE) {
            if (t.image < 0 || (uint32_t)t.image >= d->num_images) return bad("image texture references a missing image");
            continue;
        }
        return bad("unknown texture kind");
    }
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        const rtc_material& m = d->materials[i];
        if (m.kind < 0 || m.kind > 3) return bad("unknown material kind");
        if (m.kind != RTC_MAT_DIELECTRIC && (m.texture < 0 || (uint32_t)m.texture >= d->num_textures))
            return bad("material " + std::to_string(i) + " references a missing texture");
    }
    auto mat_ok = [&](int32_t m) { return m >= 0 && (uint32_t)m < d->num_materials; };
    uint64_t ntri = 0;
    for (uint32_t i = 0; i < d->num_meshes; ++i) {
        const rtc_mesh& M = d->meshes[i];
        if (!mat_ok(M.material)) return bad("mesh " + std::to_string(i) + " has a bad material");
        if (M.num_triangles && (!M.indices || !M.vertices)) return bad("mesh without vertices/indices");
        ntri += M.num_triangles;
    }
    for (uint32_t i = 0; i < d->num_spheres; ++i)
        if (!mat_ok(d->spheres[i].material) || !finite3(d->spheres[i].center) || !std::isfinite(d->spheres[i].radius))
            return bad("sphere " + std::to_string(i) + " is invalid");
    for (uint32_t i = 0; i < d->num_quads; ++i)
        if (!mat_ok(d->quads[i].material) || !finite3(d->quads[i].q) || !finite3(d->quads[i].u) || !finite3(d->quads[i].v))
            return bad("quad " + std::to_string(i) + " is invalid");
    for (uint32_t i = 0; i < d->num_omni_lights; ++i) {
        const rtc_omni_light& L = d->omni_lights[i];
        if (!finite3(L.position) || !std::isfinite(L.radius) || !finite3(L.color) || !std::isfinite(L.intensity))
            return bad("omni light " + std::to_string(i) + " is invalid");
    }
    for (uint32_t i = 0; i < d->num_spot_lights; ++i) {
        const rtc_spot_light& L = d->spot_lights[i];
        if (!finite3(L.position) || !finite3(L.direction) || !std::isfinite(L.radius) || !finite3(L.color) ||
            !std::isfinite(L.intensity) || !std::isfinite(L.cutoff) || !std::isfinite(L.falloff))
            return bad("spot light " + std::to_string(i) + " is invalid");
    }
    // transforms (1-based references, 0 = none) and boxes
    if ((d->num_transforms && !d->transforms) || (d->num_boxes && !d->boxes)) return bad("count > 0 with a null array");
    for (uint32_t i = 0; i < d->num_transforms; ++i) {
        const rtc_transform& T = d->transforms[i];
        if ((T.flags & ~7u) || !finite3(T.translate) || !finite3(T.rotate) || !finite3(T.scale))
            return bad("transform " + std::to_string(i) + " is invalid");
    }
    auto xf_ok = [&](const uint32_t* refs, uint32_t n) {
        if (!refs) return true;
        for (uint32_t i = 0; i < n; ++i)
            if (refs[i] > d->num_transforms) return false;
        return true;
    };
    if (!xf_ok(d->sphere_transforms, d->num_spheres) || !xf_ok(d->quad_transforms, d->num_quads) ||
        !xf_ok(d->mesh_transforms, d->num_meshes))
        return bad("transform reference out of range");
    for (uint32_t i = 0; i < d->num_boxes; ++i) {
        const rtc_box& B = d->boxes[i];
        if (!mat_ok(B.material) || !finite3(B.center) || !finite3(B.size) || B.transform > d->num_transforms)
            return bad("box " + std::to_string(i) + " is invalid");
    }
    auto xf_of = [](const uint32_t* refs, uint32_t i) -> int32_t { return refs ? (int32_t)refs[i] - 1 : -1; };
    // the light list: omni lights, directional lights, spot lights (load_scene, gpu.cu:504-523)
    const uint32_t n_omni = d->num_omni_lights, n_dir = d->num_dir_lights, n_spot = d->num_spot_lights;
    const uint32_t nlights = n_omni + n_dir + n_spot;
    const uint64_t nprims = (uint64_t)nlights + d->num_spheres + d->num_quads + 6ull * d->num_boxes + ntri;
    if (nprims == 0) return bad("scene has no primitives");
    if (nprims >= (1ull << 26)) return bad("scene has too many primitives (max 2^26)");
    if (d->background.kind < 0 || d->background.kind > 2) return bad("unknown background kind");
    if (d->background.kind == RTC_BG_ENV_MAP &&
        (!d->background.env_rgb || d->background.env_width <= 0 || d->background.env_height <= 0))
        return bad("environment map missing");

    // ---- primitives in global order: lights, spheres, quads, boxes, triangles -------------------
    // kind ITEM_XPRIM: a transformed sphere / quad / triangle or a box face; `inner` is then its own kind
    // (XPRIM_RECT for a face: src = box, face 0-5) and `xf` its transform (-1 for an untransformed box).
    struct PrimRef { uint8_t kind; uint8_t inner; uint8_t face; uint32_t src; int32_t xf; };
    std::vector<PrimRef> prims;
    prims.reserve(nprims);
    BvhInput bin;
    bin.boxes.reserve(nprims);
    auto sphere_light_box = [&](const float* c, float radius) {
        const float r = std::fabs(radius);
        V3 cc[2] = {v3(c[0] - r, c[1] - r, c[2] - r), v3(c[0] + r, c[1] + r, c[2] + r)};
        return box_of(cc, 2);
    };
    for (uint32_t i = 0; i < n_omni; ++i) {
        bin.boxes.push_back(sphere_light_box(d->omni_lights[i].position, d->omni_lights[i].radius));
        prims.push_back({ITEM_LIGHT, 0, 0, i, -1});
    }
    for (uint32_t i = 0; i < d->num_dir_lights; ++i) {
        const rtc_dir_light& L = d->dir_lights[i];
        V3 P = v3(L.position), U = v3(L.u), Vv = v3(L.v);
        V3 hu = mul(0.5f, U), hv = mul(0.5f, Vv);
        V3 c[4] = {sub(sub(P, hu), hv), add(sub(P, hu), hv), sub(add(P, hu), hv), add(add(P, hu), hv)};
        bin.boxes.push_back(box_of(c, 4));
        prims.push_back({ITEM_LIGHT, 0, 0, n_omni + i, -1});
    }
    for (uint32_t i = 0; i < n_spot; ++i) {
        bin.boxes.push_back(sphere_light_box(d->spot_lights[i].position, d->spot_lights[i].radius));
        prims.push_back({ITEM_LIGHT, 0, 0, n_omni + n_dir + i, -1});
    }
    for (uint32_t i = 0; i < d->num_spheres; ++i) {
        const rtc_sphere& S = d->spheres[i];
        float r = std::fabs(S.radius);
        V3 c[2] = {v3(S.center[0] - r, S.center[1] - r, S.center[2] - r), v3(S.center[0] + r, S.center[1] + r, S.center[2] + r)};
        const int32_t xi = xf_of(d->sphere_transforms, i);
        bin.boxes.push_back(xi >= 0 ? transform_box(d->transforms[xi], box_of(c, 2)) : box_of(c, 2));
        if (xi >= 0) prims.push_back({ITEM_XPRIM, ITEM_SPHERE, 0, i, xi});
        else prims.push_back({ITEM_SPHERE, 0, 0, i, -1});
    }
    for (uint32_t i = 0; i < d->num_quads; ++i) {
        const rtc_quad& Q = d->quads[i];
        V3 q = v3(Q.q), u = v3(Q.u), v = v3(Q.v);
        V3 c[4] = {q, add(q, u), add(q, v), add(add(q, u), v)};
        const int32_t xi = xf_of(d->quad_transforms, i);
        bin.boxes.push_back(xi >= 0 ? transform_box(d->transforms[xi], box_of(c, 4)) : box_of(c, 4));
        if (xi >= 0) prims.push_back({ITEM_XPRIM, ITEM_QUAD, 0, i, xi});
        else prims.push_back({ITEM_QUAD, 0, 0, i, -1});
    }
    // box faces (box.cuh:40-52): pmin = center - size / 2, pmax = pmin + size; faces front (z = pmax.z),
    // back (z = pmin.z, flipped), top (y = pmax.y), bottom (flipped), right (x = pmax.x), left (flipped)
    auto box_face = [&](const rtc_box& B, int face, float r0[4], float r1[4]) {
        float lo[3], hi[3];
        for (int k = 0; k < 3; ++k) {
            lo[k] = B.center[k] - (B.size[k] / 2.0f);
            hi[k] = lo[k] + B.size[k];
        }
        const int axis = face / 2;                    // 0 xy, 1 xz, 2 yz
        const bool low = (face & 1) != 0;
        const int a = axis == 2 ? 1 : 0, b = axis == 0 ? 1 : 2, n = axis == 0 ? 2 : axis == 1 ? 1 : 0;
        r0[0] = lo[a]; r0[1] = hi[a]; r0[2] = lo[b]; r0[3] = hi[b];
        r1[0] = low ? lo[n] : hi[n];
        r1[1] = ibits(axis);
        r1[2] = low ? 1.0f : 0.0f;
        r1[3] = ibits(B.material);
    };
    for (uint32_t i = 0; i < d->num_boxes; ++i) {
        const rtc_box& B = d->boxes[i];
        const int32_t xi = (int32_t)B.transform - 1;
        for (int f = 0; f < 6; ++f) {
            float r0[4], r1[4];
            box_face(B, f, r0, r1);
            const int axis = f / 2, a = axis == 2 ? 1 : 0, b = axis == 0 ? 1 : 2, n = axis == 0 ? 2 : axis == 1 ? 1 : 0;
            V3 c[2];
            float p0[3], p1[3];
            p0[a] = r0[0]; p1[a] = r0[1]; p0[b] = r0[2]; p1[b] = r0[3]; p0[n] = p1[n] = r1[0];
            c[0] = v3(p0[0], p0[1], p0[2]);
            c[1] = v3(p1[0], p1[1], p1[2]);
            bin.boxes.push_back(xi >= 0 ? transform_box(d->transforms[xi], box_of(c, 2)) : box_of(c, 2));
            prims.push_back({ITEM_XPRIM, (uint8_t)XPRIM_RECT, (uint8_t)f, i, xi});
        }
    }
    std::vector<uint32_t> tri_mesh;   // mesh of each flattened triangle
    std::vector<uint32_t> tri_face;
    tri_mesh.reserve(ntri);
    tri_face.reserve(ntri);
    {
        uint32_t t = 0;
        for (uint32_t m = 0; m < d->num_meshes; ++m) {
            const rtc_mesh& M = d->meshes[m];
            if (M.uvs)
                for (uint32_t k = 0; k < 2 * M.num_vertices; ++k)
                    if (!std::isfinite(M.uvs[k])) return bad("mesh " + std::to_string(m) + " texture coordinate is not finite");
            for (uint32_t f = 0; f < M.num_triangles; ++f, ++t) {
                uint32_t ia = M.indices[3 * f], ib = M.indices[3 * f + 1], ic = M.indices[3 * f + 2];
                if (ia >= M.num_vertices || ib >= M.num_vertices || ic >= M.num_vertices)
                    return bad("mesh " + std::to_string(m) + " index out of range");
                V3 c[3] = {v3(M.vertices + 3 * ia), v3(M.vertices + 3 * ib), v3(M.vertices + 3 * ic)};
                if (!finite3(M.vertices + 3 * ia) || !finite3(M.vertices + 3 * ib) || !finite3(M.vertices + 3 * ic))
                    return bad("mesh vertex is not finite");
                const int32_t xi = xf_of(d->mesh_transforms, m);
                bin.boxes.push_back(xi >= 0 ? transform_box(d->transforms[xi], box_of(c, 3)) : box_of(c, 3));
                if (xi >= 0) prims.push_back({ITEM_XPRIM, ITEM_TRI, 0, t, xi});
                else prims.push_back({ITEM_TRI, 0, 0, t, -1});
                tri_mesh.push_back(m);
                tri_face.push_back(f);
            }
        }
    }

    {
        float scale = 0.0f;
        for (int k = 0; k < 3; ++k) scale = std::max(scale, std::fabs(d->camera.look_from[k]));
        for (const Aabb& b : bin.boxes)
            for (int k = 0; k < 3; ++k) scale = std::max(scale, std::max(std::fabs(b.lo[k]), std::fabs(b.hi[k])));
        for (Aabb& b : bin.boxes) b = pad_box(b, scale);
    }

    // ---- BVH -----------------------------------------------------------------------------------
    // Transformed primitives and box faces (xprims) get a BVH of their own, walked after the main one by
    // kernels built for it; the main BVH holds every other primitive (and may be empty).
    std::vector<uint32_t> main_ids, x_ids;
    BvhInput bin_x;
    {
        BvhInput bin_main;
        for (uint32_t i = 0; i < (uint32_t)prims.size(); ++i) {
            const bool x = prims[i].kind == ITEM_XPRIM;
            (x ? x_ids : main_ids).push_back(i);
            (x ? bin_x : bin_main).boxes.push_back(bin.boxes[i]);
        }
        bin = std::move(bin_main);
    }
    BvhOutput bvh, xbvh;
    const char* berr = nullptr;
    uint32_t builder = RTC_BVH_SAH;
    if (bvh_builder != RTC_BVH_SAH && !main_ids.empty()) {
        const int rc = build_bvh_device(bin, device, bvh_builder == RTC_BVH_DEVICE_LBVH ? BVH_DEVICE_LBVH : BVH_DEVICE_PLOC,
                                        bvh, &berr);
        if (rc == BVH_DEVICE_ERROR) return fail(RTC_ERR_CUDA, std::string("device BVH build: ") + (berr ? berr : "failed"));
        if (rc == BVH_DEVICE_OK) builder = bvh_builder;
        berr = nullptr;
    }
    if (builder == RTC_BVH_SAH && !main_ids.empty() && !build_bvh(bin, 4, 0, bvh, &berr))
        return bad(berr ? berr : "BVH build failed");
    if (!x_ids.empty() && !build_bvh(bin_x, 4, 0, xbvh, &berr)) return bad(berr ? berr : "BVH build failed");
    auto t1 = std::chrono::steady_clock::now();

    // ---- materials / textures (directional lights get their own diffuse_light + solid texture) --
    std::vector<int4> tex_i;
    std::vector<float4> tex_f;
    for (uint32_t i = 0; i < d->num_textures; ++i) {
        const rtc_texture& t = d->textures[i];
        tex_i.push_back(make_int4(t.kind, t.even, t.odd, t.image));
        float inv = t.kind == RTC_TEX_CHECKER ? 1.0f / t.scale : 0.0f;   // checker_texture.cuh:23
        tex_f.push_back(make_float4(t.color[0], t.color[1], t.color[2], inv));
    }
    std::vector<int4> mat_i;
    std::vector<float4> mat_f;
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        const rtc_material& m = d->materials[i];
        float fuzz = m.fuzz < 1.0f ? m.fuzz : 1.0f;   // metal::metal (metal.cuh:52)
        mat_i.push_back(make_int4(m.kind, m.texture, 0, 0));
        mat_f.push_back(make_float4(fuzz, m.ior, m.intensity, m.directional ? 1.0f : 0.0f));
    }
    // Each light gets a solid texture of its colour and its own material, in light-list order:
    //   omni:        diffuse_light(color, intensity, directional = false)   (omni_light.cuh:13-16)
    //   directional: diffuse_light(color, intensity, directional = true)    (directional_light.cuh)
    //   spot:        diffuse_spot_light(solid(color), ...) (spot_light.cuh:47-53), kind MAT_SPOT_LIGHT,
    //                its cone read from the light record (mat_i.z = light index)
    std::vector<int32_t> light_mat(nlights);
    auto add_light_mat = [&](uint32_t li, int kind, const float* col, float intensity, float directional) {
        int32_t tex = (int32_t)tex_i.size();
        tex_i.push_back(make_int4(RTC_TEX_SOLID, 0, 0, 0));
        tex_f.push_back(make_float4(col[0], col[1], col[2], 0.0f));
        light_mat[li] = (int32_t)mat_i.size();
        mat_i.push_back(make_int4(kind, tex, (int)li, 0));
        mat_f.push_back(make_float4(0.0f, 0.0f, intensity, directional));
    };
    for (uint32_t i = 0; i < n_omni; ++i)
        add_light_mat(i, RTC_MAT_DIFFUSE_LIGHT, d->omni_lights[i].color, d->omni_lights[i].intensity, 0.0f);
    for (uint32_t i = 0; i < n_dir; ++i)
        add_light_mat(n_omni + i, RTC_MAT_DIFFUSE_LIGHT, d->dir_lights[i].color, d->dir_lights[i].intensity, 1.0f);
    for (uint32_t i = 0; i < n_spot; ++i)
        add_light_mat(n_omni + n_dir + i, MAT_SPOT_LIGHT, d->spot_lights[i].color, d->spot_lights[i].intensity, 1.0f);
    std::vector<int4> img_i;
    std::vector<uint8_t> img_bytes;
    for (uint32_t i = 0; i < d->num_images; ++i) {
        const rtc_image& im = d->images[i];
        size_t off = img_bytes.size();
        size_t nb = (size_t)im.width * im.height * 3;
        img_bytes.insert(img_bytes.end(), im.rgb, im.rgb + nb);
        img_i.push_back(make_int4((int)off, im.width, im.height, 0));
    }

    // ---- per-kind arrays in leaf order ---------------------------------------------------------
    std::vector<uint32_t> items(bvh.order.size()), xitems(xbvh.order.size());
    std::vector<float4> sph, tri, tri_n, tri_vn, tri_uv, quad, light(6 * (size_t)nlights), rect, xf;
    // per-vertex texture coordinates: when any mesh has them, every triangle gets a uv record (zeros
    // for meshes without)
    bool any_uv = false;
    for (uint32_t m = 0; m < d->num_meshes; ++m) any_uv = any_uv || d->meshes[m].uvs != nullptr;
    std::vector<int2> sph_aux;
    std::vector<int4> xprim;
    // global id bases: the lights come first, in light-list order (index = light id = global id); one id
    // per box
    const uint32_t base_sph = nlights, base_quad = base_sph + d->num_spheres, base_box = base_quad + d->num_quads,
                   base_tri = base_box + d->num_boxes;
    for (uint32_t i = 0; i < n_dir; ++i) {
        const rtc_dir_light& L = d->dir_lights[i];
        const uint32_t li = n_omni + i;
        V3 P = v3(L.position), U = v3(L.u), Vv = v3(L.v);
        PlanarPre pp = planar_pre(P, U, Vv);
        float4* q = &light[6 * (size_t)li];
        q[0] = make_float4(pp.normal.x, pp.normal.y, pp.normal.z, pp.D);
        q[1] = make_float4(P.x, P.y, P.z, ibits(light_mat[li]));
        q[2] = make_float4(U.x, U.y, U.z, ibits((int32_t)li));
        q[3] = make_float4(Vv.x, Vv.y, Vv.z, L.invisible ? 1.0f : 0.0f);
        q[4] = make_float4(pp.w.x, pp.w.y, pp.w.z, pp.area);
        q[5] = make_float4(L.color[0], L.color[1], L.color[2], L.intensity);
    }
    // sphere lights (see rtc_dev.h): q4.w < 0 marks them
    auto put_sphere_light = [&](uint32_t li, const float* pos, float radius, const float* dir, float cos_cutoff,
                                float falloff, int32_t invisible, const float* col, float intensity) {
        float4* q = &light[6 * (size_t)li];
        q[0] = make_float4(pos[0], pos[1], pos[2], radius);
        q[1] = make_float4(0.0f, 0.0f, 0.0f, ibits(light_mat[li]));
        q[2] = make_float4(dir ? dir[0] : 0.0f, dir ? dir[1] : 0.0f, dir ? dir[2] : 0.0f, ibits((int32_t)li));
        q[3] = make_float4(cos_cutoff, falloff, 0.0f, invisible ? 1.0f : 0.0f);
        q[4] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        q[5] = make_float4(col[0], col[1], col[2], intensity);
    };
    for (uint32_t i = 0; i < n_omni; ++i) {
        const rtc_omni_light& L = d->omni_lights[i];
        put_sphere_light(i, L.position, L.radius, nullptr, 0.0f, 0.0f, L.invisible, L.color, L.intensity);
    }
    for (uint32_t i = 0; i < n_spot; ++i) {
        const rtc_spot_light& L = d->spot_lights[i];
        // m_cutoff = cos(degrees_to_radians(cutoff)) (spot_light.cuh:51): degrees * M_PI / 180.0f, all float
        // (the reference's M_PI is a float literal, misc/constants.cuh:35), then the float cosine
        const float rad = L.cutoff * 3.14159265358979323846f / 180.0f;
        put_sphere_light(n_omni + n_dir + i, L.position, L.radius, L.direction, std::cos(rad), L.falloff, L.invisible,
                         L.color, L.intensity);
    }
    auto pack_sphere = [&](uint32_t src) {
        const rtc_sphere& S = d->spheres[src];
        const uint32_t typed = (uint32_t)sph.size();
        sph.push_back(make_float4(S.center[0], S.center[1], S.center[2], S.radius));
        sph_aux.push_back(make_int2(S.material, (int)(base_sph + src)));
        return typed;
    };
    auto pack_quad = [&](uint32_t src) {
        const rtc_quad& Q = d->quads[src];
        V3 q0 = v3(Q.q), u = v3(Q.u), v = v3(Q.v);
        PlanarPre pp = planar_pre(q0, u, v);
        const uint32_t typed = (uint32_t)(quad.size() / 5);
        quad.push_back(make_float4(pp.normal.x, pp.normal.y, pp.normal.z, pp.D));
        quad.push_back(make_float4(q0.x, q0.y, q0.z, ibits(Q.material)));
        quad.push_back(make_float4(u.x, u.y, u.z, ibits((int32_t)(base_quad + src))));
        quad.push_back(make_float4(v.x, v.y, v.z, 0.0f));
        quad.push_back(make_float4(pp.w.x, pp.w.y, pp.w.z, 0.0f));
        return typed;
    };
    auto pack_tri = [&](uint32_t src) {
        const rtc_mesh& M = d->meshes[tri_mesh[src]];
        uint32_t f = tri_face[src];
        uint32_t ia = M.indices[3 * f], ib = M.indices[3 * f + 1], ic = M.indices[3 * f + 2];
        V3 a = v3(M.vertices + 3 * ia), b = v3(M.vertices + 3 * ib), c = v3(M.vertices + 3 * ic);
        // triangle::triangle (triangle.cuh:87-123): v0_v1, v0_v2, middle_normal
        V3 e1 = sub(b, a), e2 = sub(c, a);
        V3 mn = unit(cross(sub(a, b), sub(a, c)));
        const uint32_t typed = (uint32_t)(tri.size() / 3);
        int32_t smooth_slot = -1;
        if (M.smooth && M.normals) {
            smooth_slot = (int32_t)(tri_vn.size() / 3);
            for (uint32_t vi : {ia, ib, ic}) {
                V3 nn = unit(v3(M.normals + 3 * vi));
                tri_vn.push_back(make_float4(nn.x, nn.y, nn.z, 0.0f));
            }
        }
        tri.push_back(make_float4(a.x, a.y, a.z, ibits(M.material)));
        tri.push_back(make_float4(e1.x, e1.y, e1.z, ibits((int32_t)(base_tri + src))));
        tri.push_back(make_float4(e2.x, e2.y, e2.z, ibits(smooth_slot)));
        tri_n.push_back(make_float4(mn.x, mn.y, mn.z, 0.0f));
        if (any_uv) {
            const float* t = M.uvs;
            auto uv = [t](uint32_t vi, int k) { return t ? t[2 * vi + k] : 0.0f; };
            tri_uv.push_back(make_float4(uv(ia, 0), uv(ia, 1), uv(ib, 0), uv(ib, 1)));
            tri_uv.push_back(make_float4(uv(ic, 0), uv(ic, 1), 0.0f, 0.0f));
        }
        return typed;
    };
    for (size_t k = 0; k < bvh.order.size() + xbvh.order.size(); ++k) {
        const bool xk = k >= bvh.order.size();
        const PrimRef& pr = xk ? prims[x_ids[xbvh.order[k - bvh.order.size()]]] : prims[main_ids[bvh.order[k]]];
        uint32_t typed = 0;
        switch (pr.kind) {
        case ITEM_LIGHT: typed = pr.src; break;
        case ITEM_SPHERE: typed = pack_sphere(pr.src); break;
        case ITEM_QUAD: typed = pack_quad(pr.src); break;
        case ITEM_TRI: typed = pack_tri(pr.src); break;
        default: {   // ITEM_XPRIM
            uint32_t inner = 0, gid = 0;
            switch (pr.inner) {
            case ITEM_SPHERE: inner = pack_sphere(pr.src); gid = base_sph + pr.src; break;
            case ITEM_QUAD: inner = pack_quad(pr.src); gid = base_quad + pr.src; break;
            case ITEM_TRI: inner = pack_tri(pr.src); gid = base_tri + pr.src; break;
            default: {
                float r0[4], r1[4];
                box_face(d->boxes[pr.src], pr.face, r0, r1);
                inner = (uint32_t)(rect.size() / 2);
                rect.push_back(make_float4(r0[0], r0[1], r0[2], r0[3]));
                rect.push_back(make_float4(r1[0], r1[1], r1[2], r1[3]));
                gid = base_box + pr.src;
            } break;
            }
            typed = (uint32_t)xprim.size();
            xprim.push_back(make_int4(pr.xf, pr.inner, (int)inner, (int)gid));
        } break;
        }
        (xk ? xitems[k - bvh.order.size()] : items[k]) = ((uint32_t)pr.kind << ITEM_KIND_SHIFT) | typed;
    }
    for (uint32_t i = 0; i < d->num_transforms; ++i) put_transform(d->transforms[i], xf);
    // the 8-wide nodes' leaf items: the same item words, regrouped per wide node
    std::vector<uint32_t> items8(bvh.items8.size());
    for (size_t k = 0; k < items8.size(); ++k) items8[k] = items[bvh.items8[k]];

    // ---- camera: perspective_camera::initialize (perspective_camera.cuh:41-108) -----------------
    DevCamera cam{};
    if (!rtc_make_camera(d->camera, cam)) return bad("degenerate camera");

    // ---- one device slab ----------------------------------------------------------------------
    struct Chunk { const void* src; size_t bytes; size_t off; };
    std::vector<Chunk> chunks;
    size_t total = 0;
    auto add_chunk = [&](const void* src, size_t bytes) {
        size_t off = total;
        chunks.push_back({src, bytes, off});
        total = align256(total + std::max<size_t>(bytes, 16));
        return off;
    };
    size_t o_nodes = add_chunk(bvh.nodes.data(), bvh.nodes.size() * sizeof(float));
    size_t o_nodes8 = add_chunk(bvh.nodes8.data(), bvh.nodes8.size() * sizeof(float));
    size_t o_items = add_chunk(items.data(), items.size() * 4);
    size_t o_items8 = add_chunk(items8.data(), items8.size() * 4);
    size_t o_sph = add_chunk(sph.data(), sph.size() * 16);
    size_t o_sphx = add_chunk(sph_aux.data(), sph_aux.size() * 8);
    size_t o_tri = add_chunk(tri.data(), tri.size() * 16);
    size_t o_trin = add_chunk(tri_n.data(), tri_n.size() * 16);
    size_t o_trivn = add_chunk(tri_vn.data(), tri_vn.size() * 16);
    size_t o_triuv = add_chunk(tri_uv.data(), tri_uv.size() * 16);
    size_t o_quad = add_chunk(quad.data(), quad.size() * 16);
    size_t o_light = add_chunk(light.data(), light.size() * 16);
    size_t o_mi = add_chunk(mat_i.data(), mat_i.size() * 16);
    size_t o_mf = add_chunk(mat_f.data(), mat_f.size() * 16);
    size_t o_ti = add_chunk(tex_i.data(), tex_i.size() * 16);
    size_t o_tf = add_chunk(tex_f.data(), tex_f.size() * 16);
    size_t o_img = add_chunk(img_i.data(), img_i.size() * 16);
    size_t o_imgb = add_chunk(img_bytes.data(), img_bytes.size());
    size_t o_xprim = add_chunk(xprim.data(), xprim.size() * 16);
    size_t o_xf = add_chunk(xf.data(), xf.size() * 16);
    size_t o_rect = add_chunk(rect.data(), rect.size() * 16);
    size_t o_xnodes = add_chunk(xbvh.nodes.data(), xbvh.nodes.size() * sizeof(float));
    size_t o_xitems = add_chunk(xitems.data(), xitems.size() * 4);
    size_t env_bytes = d->background.kind == RTC_BG_ENV_MAP
                           ? (size_t)d->background.env_width * d->background.env_height * 3 * sizeof(float) : 0;
    size_t o_env = add_chunk(env_bytes ? d->background.env_rgb : nullptr, env_bytes);
    // environment-map sampling tables (image_pdf, pdf/image_pdf.cuh:32-78): per texel luminance
    // (0.2126, 0.7152, 0.0722) x sin(theta) of its row's centre; the marginal CDF over rows, then each
    // row's conditional CDF over columns (a row of zero weight gets a uniform one)
    std::vector<float> env_cdf;
    if (env_bytes) {
        const int W = d->background.env_width, H = d->background.env_height;
        const float* px = d->background.env_rgb;
        env_cdf.assign((size_t)H + (size_t)W * H, 0.0f);
        std::vector<double> row(H, 0.0);
        double total = 0.0;
        for (int y = 0; y < H; ++y) {
            const double st = std::sin(3.14159265358979323846 * (1.0 - (y + 0.5) / H));
            double acc = 0.0;
            float* C = env_cdf.data() + H + (size_t)y * W;
            for (int x = 0; x < W; ++x) {
                const float* q = px + 3 * ((size_t)y * W + x);
                acc += std::max(0.0, (0.2126 * q[0] + 0.7152 * q[1] + 0.0722 * q[2]) * st);
                C[x] = (float)acc;
            }
            for (int x = 0; x < W; ++x) C[x] = acc > 0.0 ? (float)(C[x] / acc) : (float)(x + 1) / (float)W;
            C[W - 1] = 1.0f;
            row[y] = acc;
            total += acc;
        }
        double acc = 0.0;
        for (int y = 0; y < H; ++y) {
            acc += row[y];
            env_cdf[y] = total > 0.0 ? (float)(acc / total) : 0.0f;
        }
        if (total > 0.0) env_cdf[H - 1] = 1.0f;
        else env_cdf.clear();   // a black map: nothing to sample
    }
    size_t o_envcdf = add_chunk(env_cdf.data(), env_cdf.size() * sizeof(float));

    // host image of the device slab; the DevScene's pointer fields hold byte offsets into it
    H.slab.assign(total, 0);
    for (const Chunk& c : chunks)
        if (c.src && c.bytes) std::memcpy(H.slab.data() + c.off, c.src, c.bytes);
    auto off = [](size_t o) { return reinterpret_cast<uint8_t*>(static_cast<uintptr_t>(o)); };
    DevScene& D = H.dev;
    D = DevScene{};
    D.nodes = (const float4*)off(o_nodes);
    D.nodes8 = bvh.num_nodes8 ? (const float4*)off(o_nodes8) : nullptr;
    D.items = (const uint32_t*)off(o_items);
    D.items8 = bvh.num_nodes8 ? (const uint32_t*)off(o_items8) : nullptr;
    D.sph = (const float4*)off(o_sph);
    D.sph_aux = (const int2*)off(o_sphx);
    D.tri = (const float4*)off(o_tri);
    D.tri_n = (const float4*)off(o_trin);
    D.tri_vn = (const float4*)off(o_trivn);
    D.tri_uv = tri_uv.empty() ? nullptr : (const float4*)off(o_triuv);
    D.quad = (const float4*)off(o_quad);
    D.light = (const float4*)off(o_light);
    D.mat_i = (const int4*)off(o_mi);
    D.mat_f = (const float4*)off(o_mf);
    D.tex_i = (const int4*)off(o_ti);
    D.tex_f = (const float4*)off(o_tf);
    D.images = (const int4*)off(o_img);
    D.image_bytes = (const uint8_t*)off(o_imgb);
    D.xprim = (const int4*)off(o_xprim);
    D.xf = (const float4*)off(o_xf);
    D.rect = (const float4*)off(o_rect);
    D.num_xprim = (uint32_t)xprim.size();
    D.num_xf = d->num_transforms;
    D.num_rect = (uint32_t)(rect.size() / 2);
    D.xnodes = xbvh.num_nodes ? (const float4*)off(o_xnodes) : nullptr;
    D.xitems = xbvh.num_nodes ? (const uint32_t*)off(o_xitems) : nullptr;
    D.num_xnodes = xbvh.num_nodes;
    D.num_xitems = (uint32_t)xitems.size();
    D.num_nodes = bvh.num_nodes;
    D.num_nodes8 = bvh.num_nodes8;
    D.num_items = (uint32_t)items.size();
    D.num_lights = nlights;
    D.num_materials = (uint32_t)mat_i.size();
    D.num_textures = (uint32_t)tex_i.size();
    D.num_images = (uint32_t)img_i.size();
    D.num_sph = (uint32_t)sph.size();
    D.num_tri = (uint32_t)tri_n.size();
    D.num_quad = (uint32_t)(quad.size() / 5);
    D.cam = cam;
    D.bg.kind = d->background.kind;
    for (int k = 0; k < 3; ++k) { D.bg.color[k] = d->background.color[k]; D.bg.top[k] = d->background.top[k]; }
    D.bg.env = env_bytes ? (const float*)off(o_env) : nullptr;
    D.bg.env_w = d->background.env_width;
    D.bg.env_h = d->background.env_height;
    D.bg.cdf = env_cdf.empty() ? nullptr : (const float*)off(o_envcdf);
    D.bg.pdf_scale = env_cdf.empty() ? 0.0f
                                     : (float)((double)D.bg.env_w * D.bg.env_h /
                                               (2.0 * 3.14159265358979323846 * 3.14159265358979323846));
    H.cam = d->camera;
    H.info = rtc_scene_info{};
    H.info.num_primitives = (uint32_t)nprims;
    H.info.num_lights = nlights;
    H.info.num_nodes = bvh.num_nodes;
    H.info.max_leaf_size = bvh.max_leaf_seen;
    H.info.device_bytes = total;
    H.info.build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    H.info.bvh_builder = builder;
    H.info.num_wide_nodes = bvh.num_nodes8;
    return RTC_OK;
}

DevScene rtc_rebase_scene(const HostScene& H, uint8_t* base) {
    DevScene D = H.dev;
    auto rb = [base](auto& p) {
        p = reinterpret_cast<std::remove_reference_t<decltype(p)>>(base + reinterpret_cast<uintptr_t>(p));
    };
    rb(D.nodes);
    rb(D.items);
    if (D.nodes8) { rb(D.nodes8); rb(D.items8); }
    rb(D.sph); rb(D.sph_aux); rb(D.tri); rb(D.tri_n); rb(D.tri_vn); rb(D.quad);
    rb(D.light); rb(D.mat_i); rb(D.mat_f); rb(D.tex_i); rb(D.tex_f); rb(D.images); rb(D.image_bytes);
    rb(D.xprim); rb(D.xf); rb(D.rect);
    if (D.xnodes) { rb(D.xnodes); rb(D.xitems); }
    if (D.bg.env) rb(D.bg.env);
    if (D.bg.cdf) rb(D.bg.cdf);
    if (D.tri_uv) rb(D.tri_uv);
    return D;
}

extern "C" rtc_status rtc_scene_create(rtc_context* ctx, const rtc_scene_desc* d, rtc_scene** out) {
    return rtc_scene_create_ex(ctx, d, nullptr, out);
}

extern "C" rtc_status rtc_scene_create_ex(rtc_context* ctx, const rtc_scene_desc* d, const rtc_scene_options* opt,
                                          rtc_scene** out) {
    if (!ctx || !d || !out) return fail(RTC_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (opt && (opt->reserved[0] || opt->reserved[1] || opt->reserved[2]))
        return fail(RTC_ERR_INVALID_ARGUMENT, "reserved scene options must be zero");
    HostScene H;
    rtc_status r = rtc_build_host_scene(d, H, opt ? opt->bvh_builder : RTC_BVH_SAH, ctx->device);
    if (r != RTC_OK) return r;
    rtc_scene* s = new (std::nothrow) rtc_scene();
    if (!s) return fail(RTC_ERR_OOM, "host allocation failed");
    s->ctx = ctx;
    s->device = ctx->device;
    RtcDeviceScope dev(ctx->device);
    const size_t total = H.slab.size();
    cudaError_t e = cudaMalloc(&s->d_slab, total);
    if (e != cudaSuccess) { delete s; return cuda_fail(e, "cudaMalloc(scene)"); }
    s->slab_bytes = total;
    e = cudaMemcpyAsync(s->d_slab, H.slab.data(), total, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { cudaFree(s->d_slab); delete s; return cuda_fail(e, "scene upload"); }
    s->dev = rtc_rebase_scene(H, (uint8_t*)s->d_slab);
    s->cam = H.cam;
    s->info = H.info;
    *out = s;
    return RTC_OK;
}

extern "C" rtc_status rtc_scene_destroy(rtc_scene* s) {
    // A scene may outlive its context: only its own device id is used here (cudaFree synchronises
    // with the device before releasing the memory).
    if (!s) return RTC_OK;
    RtcDeviceScope dev(s->device);
    cudaFree(s->d_slab);
    delete s;
    return RTC_OK;
}

extern "C" rtc_status rtc_scene_get_info(const rtc_scene* s, rtc_scene_info* info) {
    if (!s || !info) return fail(RTC_ERR_INVALID_ARGUMENT, "null argument");
    *info = s->info;
    return RTC_OK;
}

// ---------------------------------------------------------------------------------------------------
// render
// ---------------------------------------------------------------------------------------------------
namespace {

rtc_status check_params(const rtc_render_params* p) {
    if (!p) return fail(RTC_ERR_INVALID_ARGUMENT, "params is null");
    if (p->width <= 0 || p->height <= 0) return fail(RTC_ERR_INVALID_ARGUMENT, "width/height must be positive");
    if ((int64_t)p->width * p->height > (1ll << 31)) return fail(RTC_ERR_INVALID_ARGUMENT, "image too large");
    if (p->spp <= 0) return fail(RTC_ERR_INVALID_ARGUMENT, "spp must be positive");
    if (p->max_depth <= 0 || p->max_depth > WF_MAX_DEPTH) return fail(RTC_ERR_INVALID_ARGUMENT, "max_depth out of range (1..65535)");
    if (p->mode != RTC_MODE_COMPAT && p->mode != RTC_MODE_CLEAN) return fail(RTC_ERR_INVALID_ARGUMENT, "unknown mode");
    if (p->draw_order != RTC_DRAW_ORDER_DEVICE && p->draw_order != RTC_DRAW_ORDER_HOST)
        return fail(RTC_ERR_INVALID_ARGUMENT, "unknown draw order");
    if (p->engine < RTC_ENGINE_AUTO || p->engine > RTC_ENGINE_WAVEFRONT)
        return fail(RTC_ERR_INVALID_ARGUMENT, "unknown engine");
    return RTC_OK;
}

DevParams dev_params(const rtc_render_params* p) { return rtc_dev_params(p); }

}  // namespace

DevParams rtc_dev_params(const rtc_render_params* p) {
    DevParams P;
    P.width = p->width;
    P.height = p->height;
    P.spp = p->spp;
    P.sqrt_spp = (int)std::sqrt((double)p->spp);   // gpu.cu:1989
    P.max_depth = p->max_depth;
    P.seed = p->seed;
    P.draw_order = p->draw_order;
    P.num_pixels = (int64_t)p->width * p->height;
    P.groups = (p->mode == RTC_MODE_CLEAN && (p->flags & RTC_FLAG_SAMPLE_GROUPS)) ? std::min(8, p->spp) : 1;
    P.rgb8 = nullptr;
    return P;
}

size_t rtc_group_bytes(const rtc_render_params* p) {
    const DevParams P = rtc_dev_params(p);
    if (P.groups <= 1) return 0;
    const size_t npix = (size_t)P.num_pixels;
    return ((npix * (size_t)P.groups * sizeof(float4) + 255) & ~(size_t)255) + npix * sizeof(uint32_t);
}

void rtc_carve_groups(void* base, const rtc_render_params* p, float4** part, uint32_t** gcnt) {
    const DevParams P = rtc_dev_params(p);
    const size_t npix = (size_t)P.num_pixels;
    *part = (float4*)base;
    *gcnt = (uint32_t*)((uint8_t*)base + ((npix * (size_t)P.groups * sizeof(float4) + 255) & ~(size_t)255));
}

namespace {

// Bytes of wavefront scratch per path slot.
constexpr size_t WF_SLOT_BYTES = WF_REC_BYTES + 3 * sizeof(uint32_t);
constexpr uint32_t WF_MAX_SLOTS = 1u << 22;   // 4,194,304 slots = 432 MiB of path state (108 B per slot)

// Lays out the wavefront buffers for `slots` path slots in one block of device memory at `base`
// (the context's scratch, or the allocation-free entry point's static array).
size_t carve_wavefront(void* base, uint32_t slots, WfBuffers& B) {
    uint8_t* p = (uint8_t*)base;
    auto take = [&](size_t bytes) {
        uint8_t* r = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void*)r;
    };
    const size_t n = slots;
    B.rec = (uint32_t*)take(n * WF_REC_BYTES);
    B.queue[0] = (uint32_t*)take(n * 4);
    B.queue[1] = (uint32_t*)take(n * 4);
    B.queue[2] = (uint32_t*)take(n * 4);
    B.ctr = (uint32_t*)take(WF_CTR_N * 4);
    B.slots = slots;
    return (size_t)(p - (uint8_t*)base);
}

}  // namespace

bool rtc_dynamic_chunks(bool fallback) {
    static const int v = [] {
        const char* ev = std::getenv("RTC_WF_DYNAMIC");
        return ev ? (std::atoi(ev) != 0 ? 1 : 0) : -1;
    }();
    return v >= 0 ? v != 0 : fallback;
}

int rtc_drain_every(int fallback) {
    static const int every = [] {
        const char* ev = std::getenv("RTC_WF_DRAIN_EVERY");
        return ev ? std::max(0, std::atoi(ev)) : -1;
    }();
    return every >= 0 ? every : fallback;
}

namespace {

// Bytes carve_wavefront lays out for `slots` slots (each buffer rounded up to 256 bytes).
constexpr size_t wavefront_bytes(size_t n) {
    return ((n * WF_REC_BYTES + 255) & ~(size_t)255) + 3 * ((n * 4 + 255) & ~(size_t)255) +
           ((WF_CTR_N * 4 + 255) & ~(size_t)255);
}
// The allocation-free render's advertised cap fits its 64 MiB array behind a 256-byte status header
// (render_noalloc.cu), so an image at or under RTC_NOALLOC_MAX_PIXELS never fails for lack of room.
static_assert(256 + wavefront_bytes(RTC_NOALLOC_MAX_PIXELS) <= (size_t(64) << 20),
              "RTC_NOALLOC_MAX_PIXELS slots do not fit the allocation-free render's static array");
static_assert(wavefront_bytes(1) <= WF_SLOT_BYTES + 12 * 256, "wavefront layout grew past WF_SLOT_BYTES");

rtc_status ensure_wavefront(rtc_context* c, uint32_t slots, WfBuffers& B) {
    if (c->wf_cap < slots) {
        cudaFree(c->d_wf);
        c->d_wf = nullptr;
        c->wf_cap = 0;
        size_t bytes = (size_t)slots * WF_SLOT_BYTES + 16 * 256;
        RTC_CUDA(cudaMalloc(&c->d_wf, bytes));
        c->wf_cap = slots;
    }
    if (!c->h_poll) {
        RTC_CUDA(cudaMallocHost(&c->h_poll, 2 * sizeof(uint32_t)));
        RTC_CUDA(cudaEventCreateWithFlags(&c->poll_ev[0], cudaEventDisableTiming));
        RTC_CUDA(cudaEventCreateWithFlags(&c->poll_ev[1], cudaEventDisableTiming));
        for (cudaEvent_t& e : c->phase_ev) RTC_CUDA(cudaEventCreate(&e));
        for (cudaEvent_t& e : c->split_ev) RTC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        RTC_CUDA(cudaStreamCreateWithFlags(&c->stream_long, cudaStreamNonBlocking));
    }
    carve_wavefront(c->d_wf, slots, B);
    return RTC_OK;
}

// How the host learns the queue size after a batch of iterations.
struct WfPoller {
    uint32_t* h = nullptr;           // pinned slots: the next batch is queued before the host looks
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool sync = false;               // synchronous copy into a host variable (no pinned memory, no events)
    // long-chain split: the stream its drain kernel runs on (null: the render's own stream, in order)
    // and the two events that order it (split done -> long chains start; long chains done -> render end)
    cudaStream_t st_long = nullptr;
    cudaEvent_t split_ev[2] = {nullptr, nullptr};
};

struct WfRun {
    uint64_t iterations = 0;
    bool drained = false;
    uint32_t drained_slots = 0;
    bool split = false;
};

// Wavefront engine: init, then batches of (extend, shade) iterations until the slot queue drains or
// falls under the drain threshold, where one finish launch completes the remaining slots.
// Optional per-launch timing: event pairs around extend launches (first half of the pool order) and
// shade launches, created on demand.
struct WfTimer {
    std::vector<cudaEvent_t>* pool = nullptr;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ext, shade;
    size_t used = 0;
    cudaError_t pair(cudaEvent_t& a, cudaEvent_t& b) {
        while (pool->size() < used + 2) {
            cudaEvent_t e;
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) return r;
            pool->push_back(e);
        }
        a = (*pool)[used];
        b = (*pool)[used + 1];
        used += 2;
        return cudaSuccess;
    }
};

// `xp`: the scene has transformed primitives or boxes (an xprim BVH), walked by the RTC_XP=1 kernels.
rtc::WfOneFn wf_one_fn(const rtc_render_params* p, bool xp) {
    if (p->mode == RTC_MODE_CLEAN) return xp ? rtc_wf_one_clean_x : rtc_wf_one_clean;
    if (p->draw_order == RTC_DRAW_ORDER_HOST) return xp ? rtc_wf_one_compat_host_x : rtc_wf_one_compat_host;
    return xp ? rtc_wf_one_compat_dev_x : rtc_wf_one_compat_dev;
}

rtc_status run_wavefront(const DevScene& S, const rtc_render_params* p, const WfBuffers& B, uint32_t* d_status,
                         float4* d_out, unsigned long long* d_counters, cudaStream_t st, int num_sms,
                         const WfPoller& poll, cudaEvent_t* phase, WfRun& run, WfTimer* timer = nullptr,
                         void* groups = nullptr, uint8_t* d_rgb8 = nullptr) {
    DevParams P = dev_params(p);
    P.rgb8 = d_rgb8;   // quantised output written as each pixel finishes
    const bool clean = p->mode == RTC_MODE_CLEAN;
    const WfOneFn fn = wf_one_fn(p, S.num_xnodes != 0);
    WfOneArgs J;
    J.S = S;
    J.P = P;
    J.out = d_out;
    J.part = nullptr;
    J.gcnt = nullptr;
    if (P.groups > 1) {
        if (!groups) return fail(RTC_ERR_INVALID_ARGUMENT, "sample groups need scratch memory");
        rtc_carve_groups(groups, p, &J.part, &J.gcnt);
        RTC_CUDA(cudaMemsetAsync(J.gcnt, 0, (size_t)P.num_pixels * sizeof(uint32_t), st));
    }
    WfLaunch L{};
    L.counters = d_counters;
    L.status = d_status;
    L.st = st;
    L.wide = S.nodes8 != nullptr;
    if (phase) RTC_CUDA(cudaEventRecord(phase[0], st));
    RTC_CUDA(cudaMemsetAsync(B.ctr, 0, WF_CTR_N * sizeof(uint32_t), st));
    const int grid = num_sms * 8;
    L.grid = (int)std::min<int64_t>((B.slots + 127) / 128, (int64_t)num_sms * 16);
    cudaError_t e = fn(WF_OP_INIT, J, B, L);
    if (e != cudaSuccess) return cuda_fail(e, "wavefront init");
    L.grid = grid;
    const uint64_t nsamp = clean ? (uint64_t)P.spp : (uint64_t)P.sqrt_spp * P.sqrt_spp;
    const uint64_t rounds = (uint64_t)((P.num_pixels * P.groups + B.slots - 1) / B.slots);
    const uint64_t max_iters = rounds * nsamp * (uint64_t)(P.max_depth + 1) + 64;
    const int BATCH = 8;
    // drain threshold: below this many queued slots the finish kernel takes over
    uint32_t drain = (uint32_t)num_sms * 512u;
    if (const char* ev = std::getenv("RTC_WF_DRAIN")) drain = (uint32_t)std::strtoul(ev, nullptr, 10);
    // Drain kernel: one thread per slot for its whole chain, or the compacting drain, whose live slots
    // are repacked into full warps every 2 bounce steps.  A frame with fewer work units than the drain
    // threshold runs almost whole in the drain, where its short chains leave the lanes idle: there the
    // compacting drain pays (Cornell 256x256, 16 spp: drain 1.91 -> 1.52 ms).  In a larger frame the
    // drain is bound by its longest chains' bounce latency, which packing does not shorten (spheres
    // frame: 19.0 against 18.6-19.4 ms), and its barriers cost a DRAM-bound walk (meshes frame: 67.7
    // against 98.9 ms), so it keeps the plain drain.
    L.drain_every = rtc_drain_every(P.num_pixels * (int64_t)P.groups <= (int64_t)drain ? 2 : 0);
    // Queue chunks handed out by a counter for scenes of 2^20 primitives or more, whose walks are long
    // and uneven (meshes frame, 1.31 M triangles: extend 450.7 -> 405.5 ms, 436 -> 460-467 Mpaths/s);
    // the fixed grid stride for smaller ones (spheres frame, 489 primitives: 945 against 840 Mpaths/s;
    // the 64 batch scenes of up to 500 K triangles, one image per call: 631 against 608 in compat mode,
    // 1,167 against 1,001 in clean mode with sample groups).
    L.dynamic = rtc_dynamic_chunks(S.num_items >= (1u << 20));
    // long-chain split: at iteration `split_at` (0: never), slots predicted to need more than
    // `split_thr` further iterations move to the drain kernel, running beside the bulk iterations
    uint64_t split_at = 0;
    float split_thr = 1024.0f;
    if (const char* ev = std::getenv("RTC_WF_SPLIT")) split_at = std::strtoull(ev, nullptr, 10);
    if (const char* ev = std::getenv("RTC_WF_SPLIT_THRESH")) split_thr = std::strtof(ev, nullptr);
    int split_blocks = 1;   // blocks per SM of the long-chain kernel (its registers stay taken while it runs)
    if (const char* ev = std::getenv("RTC_WF_SPLIT_BLOCKS")) split_blocks = std::max(1, std::atoi(ev));
    int64_t last_left = -1;   // queue size last observed (one batch late in both polling modes)
    // split extend / shade kernels (default) or one fused launch per iteration
    bool fused = false;
    if (const char* ev = std::getenv("RTC_WF_FUSED")) fused = std::atoi(ev) != 0;
    uint64_t it = 0;
    int pending = -1;   // poll slot of the previous batch
    uint32_t left = 0;
    uint32_t sync_counts[2] = {0, 0};
    // Copies the queue size after the batch just enqueued and reads the previous batch's (lagged).
    auto poll_batch = [&](int b, bool& have) -> rtc_status {
        const int slot = b & 1;
        if (poll.sync) {
            uint32_t h = 0;
            RTC_CUDA(cudaMemcpyAsync(&h, B.ctr + wf_iter(it).cin, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            RTC_CUDA(cudaStreamSynchronize(st));
            sync_counts[slot] = h;
            if (pending >= 0) {
                left = sync_counts[pending];
                have = true;
            }
        } else {
            RTC_CUDA(cudaMemcpyAsync(poll.h + slot, B.ctr + wf_iter(it).cin, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                     st));
            RTC_CUDA(cudaEventRecord(poll.ev[slot], st));
            if (pending >= 0) {
                RTC_CUDA(cudaEventSynchronize(poll.ev[pending]));
                left = poll.h[pending];
                have = true;
            }
        }
        pending = slot;
        return RTC_OK;
    };
    for (int b = 0;; ++b) {
        if (!run.split && split_at > 0 && it >= split_at && last_left >= (int64_t)drain) {
            // the split takes the place of one iteration (same queue rotation)
            L.w = wf_iter(it);
            L.k0 = (float)it;
            L.threshold = split_thr;
            e = fn(WF_OP_SPLIT, J, B, L);
            if (e != cudaSuccess) return cuda_fail(e, "wavefront split");
            ++it;
            run.split = true;
            WfLaunch LL = L;
            LL.w = WfIter{2, WF_LONG, 0, 0};
            LL.grid = num_sms * split_blocks;
            LL.st = poll.st_long ? poll.st_long : st;
            if (poll.st_long) {
                RTC_CUDA(cudaEventRecord(poll.split_ev[0], st));
                RTC_CUDA(cudaStreamWaitEvent(poll.st_long, poll.split_ev[0], 0));
            }
            e = fn(WF_OP_FINISH, J, B, LL);
            if (e != cudaSuccess) return cuda_fail(e, "wavefront long chains");
            if (poll.st_long) RTC_CUDA(cudaEventRecord(poll.split_ev[1], poll.st_long));
        }
        for (int k = 0; k < BATCH; ++k, ++it) {
            L.w = wf_iter(it);
            if (fused) {
                e = fn(WF_OP_BOUNCE, J, B, L);
            } else {
                cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
                if (timer) {
                    RTC_CUDA(timer->pair(e0, e1));
                    RTC_CUDA(timer->pair(e2, e3));
                    RTC_CUDA(cudaEventRecord(e0, st));
                }
                e = fn(WF_OP_EXTEND, J, B, L);
                if (timer) {
                    RTC_CUDA(cudaEventRecord(e1, st));
                    RTC_CUDA(cudaEventRecord(e2, st));
                    timer->ext.push_back({e0, e1});
                }
                if (e == cudaSuccess) e = fn(WF_OP_SHADE, J, B, L);
                if (timer) {
                    RTC_CUDA(cudaEventRecord(e3, st));
                    timer->shade.push_back({e2, e3});
                }
            }
            if (e != cudaSuccess) return cuda_fail(e, "wavefront iteration");
        }
        // Both polling modes act on the count of the PREVIOUS batch (the next batch is already
        // queued when the host looks), so the drain point - and with it the result - does not depend
        // on the polling mode.
        bool have = false;
        rtc_status pr = poll_batch(b, have);
        if (pr != RTC_OK) return pr;
        if (have) last_left = (int64_t)left;
        if (have && left == 0) break;
        if (have && left < drain) {
            run.drained = true;
            break;
        }
        if (it > max_iters) return fail(RTC_ERR_TIMEOUT, "wavefront did not drain within its iteration bound");
    }
    run.iterations = it;
    run.drained_slots = run.drained ? left : 0u;
    if (phase) RTC_CUDA(cudaEventRecord(phase[1], st));
    if (run.drained) {
        L.w = wf_iter(it);
        const uint32_t per_block = L.drain_every > 0 ? (uint32_t)rtc::WF_DRAIN_BLOCK : 128u;
        L.grid = (int)std::max<uint32_t>(1u, (drain + per_block - 1u) / per_block);
        e = fn(WF_OP_FINISH, J, B, L);
        if (e != cudaSuccess) return cuda_fail(e, "wavefront finish");
    }
    if (run.split && poll.st_long) RTC_CUDA(cudaStreamWaitEvent(st, poll.split_ev[1], 0));   // long chains done
    if (phase) RTC_CUDA(cudaEventRecord(phase[2], st));
    return RTC_OK;
}

rtc_status launch_wavefront(rtc_context* c, const rtc_scene* s, const rtc_render_params* p, float4* d_out,
                            unsigned long long* d_counters, cudaStream_t st, uint8_t* d_rgb8) {
    const int64_t units = (int64_t)p->width * p->height * dev_params(p).groups;
    const uint32_t slots = (uint32_t)std::min<int64_t>(units, WF_MAX_SLOTS);
    WfBuffers B;
    rtc_status r = ensure_wavefront(c, slots, B);
    if (r != RTC_OK) return r;
    const size_t gbytes = rtc_group_bytes(p);
    if (gbytes > c->groups_cap) {
        cudaFree(c->d_groups);
        c->d_groups = nullptr;
        c->groups_cap = 0;
        RTC_CUDA(cudaMalloc(&c->d_groups, gbytes));
        c->groups_cap = gbytes;
    }
    WfPoller poll;
    poll.h = c->h_poll;
    poll.ev[0] = c->poll_ev[0];
    poll.ev[1] = c->poll_ev[1];
    poll.st_long = c->stream_long;
    poll.split_ev[0] = c->split_ev[0];
    poll.split_ev[1] = c->split_ev[1];
    WfRun run;
    WfTimer timer;
    timer.pool = &c->kev;
    const bool timed = (p->flags & RTC_FLAG_KERNEL_TIMING) != 0;
    r = run_wavefront(rtc_scene_view(s, p), p, B, c->d_status, d_out, d_counters, st, c->num_sms, poll,
                      c->phase_ev, run, timed ? &timer : nullptr, c->d_groups, d_rgb8);
    if (r != RTC_OK) return r;
    c->kev_ext = c->kev_shade = 0;
    c->kev_pairs.clear();
    if (timed) {
        c->kev_ext = (uint32_t)timer.ext.size();
        c->kev_shade = (uint32_t)timer.shade.size();
        for (auto& pr : timer.ext) c->kev_pairs.push_back(pr);
        for (auto& pr : timer.shade) c->kev_pairs.push_back(pr);
    }
    const bool fused = std::getenv("RTC_WF_FUSED") && std::atoi(std::getenv("RTC_WF_FUSED")) != 0;
    c->last = rtc_render_stats{};
    c->last.engine = RTC_ENGINE_WAVEFRONT;
    c->last.iterations = (uint32_t)run.iterations;
    // (the split pass counts as one iteration: the split launch and the long-chain drain launch)
    c->last.launches = (uint32_t)(1 + (fused ? 1 : 2) * run.iterations + (run.drained ? 1 : 0));
    c->last.drained_slots = run.drained_slots;
    c->last_timed = true;
    return RTC_OK;
}

}  // namespace

// ---- internal helpers shared with render_noalloc.cu (rtc_internal.h) ----
size_t rtc_wf_slot_bytes() { return WF_SLOT_BYTES; }
size_t rtc_carve_wavefront(void* base, uint32_t slots, WfBuffers& B) { return carve_wavefront(base, slots, B); }
rtc_status rtc_set_error(rtc_status s, const char* msg) { return fail(s, msg); }
rtc_status rtc_check_render_params(const rtc_render_params* p) { return check_params(p); }
int rtc_scene_device(const rtc_scene* s) { return s->device; }
rtc_status rtc_run_wavefront_sync(const rtc_scene* s, const rtc_render_params* p, const WfBuffers& B,
                                  uint32_t* d_status, float4* d_out, cudaStream_t st) {
    int dev = 0, sms = 148;
    RTC_CUDA(cudaGetDevice(&dev));
    RTC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    WfPoller poll;
    poll.sync = true;
    WfRun run;
    return run_wavefront(rtc_scene_view(s, p), p, B, d_status, d_out, nullptr, st, sms, poll, nullptr, run);
}

namespace {

// d_rgb8 (may be null): the quantised, row-flipped RGB8 image, written by the render kernels as each
// pixel finishes (prepare_pixel_color + the output loop fused into the accumulation).
rtc_status launch(rtc_context* c, const rtc_scene* s, const rtc_render_params* p, float4* d_out,
                  unsigned long long* d_counters, cudaStream_t st, uint8_t* d_rgb8) {
    if (p->engine != RTC_ENGINE_MEGAKERNEL) return launch_wavefront(c, s, p, d_out, d_counters, st, d_rgb8);
    c->last = rtc_render_stats{};
    c->last.engine = RTC_ENGINE_MEGAKERNEL;
    c->last.launches = 1;
    c->last_timed = false;
    DevParams P = dev_params(p);
    P.rgb8 = d_rgb8;
    const DevScene S = rtc_scene_view(s, p);
    const bool xp = S.num_xnodes != 0;
    auto fn = p->mode == RTC_MODE_CLEAN ? (xp ? rtc_launch_render_clean_x : rtc_launch_render_clean)
              : p->draw_order == RTC_DRAW_ORDER_HOST ? (xp ? rtc_launch_render_compat_host_x : rtc_launch_render_compat_host)
                                                     : (xp ? rtc_launch_render_compat_dev_x : rtc_launch_render_compat_dev);
    cudaError_t e = fn(S, P, d_out, d_counters, c->d_status, p->block_size, st);
    if (e != cudaSuccess) return cuda_fail(e, "render launch");
    return RTC_OK;
}

rtc_status read_status(rtc_context* c) {
    uint32_t st = 0;
    RTC_CUDA(cudaMemcpyAsync(&st, c->d_status, 4, cudaMemcpyDeviceToHost, c->stream));
    RTC_CUDA(cudaStreamSynchronize(c->stream));
    if (st) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "kernel status word 0x%x (1=stack 2=item 4=material 8=texture 16=timeout)", st);
        return fail((st & STATUS_TIMEOUT) ? RTC_ERR_TIMEOUT : RTC_ERR_DEVICE_CHECK, buf);
    }
    return RTC_OK;
}

}  // namespace

extern "C" rtc_status rtc_render(rtc_context* c, const rtc_scene* s, const rtc_render_params* p, float* radiance_sum,
                                 uint8_t* rgb8) {
    if (!c || !s) return fail(RTC_ERR_INVALID_ARGUMENT, "null context/scene");
    rtc_status r = check_params(p);
    if (r != RTC_OK) return r;
    std::lock_guard<std::mutex> lk(c->mu);
    RtcDeviceScope dev(c->device);
    RTC_CUDA(dev.error());
    const size_t npix = (size_t)p->width * p->height;
    if (c->out_cap < npix) {
        cudaFree(c->d_out);
        c->d_out = nullptr;
        c->out_cap = 0;
        RTC_CUDA(cudaMalloc(&c->d_out, npix * sizeof(float4)));
        c->out_cap = npix;
    }
    if (rgb8 && c->rgb8_cap < npix * 3) {
        cudaFree(c->d_rgb8);
        c->d_rgb8 = nullptr;
        c->rgb8_cap = 0;
        RTC_CUDA(cudaMalloc(&c->d_rgb8, npix * 3));
        c->rgb8_cap = npix * 3;
    }
    RTC_CUDA(cudaMemsetAsync(c->d_status, 0, 4, c->stream));
    r = launch(c, s, p, c->d_out, nullptr, c->stream, rgb8 ? c->d_rgb8 : nullptr);
    if (r != RTC_OK) return r;
    if (rgb8) RTC_CUDA(cudaMemcpyAsync(rgb8, c->d_rgb8, npix * 3, cudaMemcpyDeviceToHost, c->stream));
    if (radiance_sum)
        RTC_CUDA(cudaMemcpyAsync(radiance_sum, c->d_out, npix * sizeof(float4), cudaMemcpyDeviceToHost, c->stream));
    RTC_CUDA(cudaStreamSynchronize(c->stream));
    return read_status(c);
}

extern "C" rtc_status rtc_render_device(rtc_context* c, const rtc_scene* s, const rtc_render_params* p,
                                        float* d_radiance_sum, uint8_t* d_rgb8, unsigned long long* d_counters,
                                        void* stream) {
    if (!c || !s || !d_radiance_sum) return fail(RTC_ERR_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)d_radiance_sum & 15u) != 0) return fail(RTC_ERR_INVALID_ARGUMENT, "radiance buffer must be 16-byte aligned");
    rtc_status r = check_params(p);
    if (r != RTC_OK) return r;
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    RtcDeviceScope dev(c->device);
    RTC_CUDA(dev.error());
    return launch(c, s, p, (float4*)d_radiance_sum, d_counters, st, d_rgb8);
}

extern "C" rtc_status rtc_get_render_stats(rtc_context* c, rtc_render_stats* out) {
    if (!c || !out) return fail(RTC_ERR_INVALID_ARGUMENT, "null argument");
    *out = c->last;
    if (c->last_timed) {
        RTC_CUDA(cudaEventSynchronize(c->phase_ev[2]));
        RTC_CUDA(cudaEventElapsedTime(&out->bulk_ms, c->phase_ev[0], c->phase_ev[1]));
        RTC_CUDA(cudaEventElapsedTime(&out->drain_ms, c->phase_ev[1], c->phase_ev[2]));
        out->extend_launches = c->kev_ext;
        out->shade_launches = c->kev_shade;
        for (uint32_t i = 0; i < c->kev_ext + c->kev_shade; ++i) {
            float ms = 0.f;
            RTC_CUDA(cudaEventElapsedTime(&ms, c->kev_pairs[i].first, c->kev_pairs[i].second));
            if (i < c->kev_ext) out->extend_ms += ms;
            else out->shade_ms += ms;
        }
    }
    return RTC_OK;
}

extern "C" rtc_status rtc_trace_closest(rtc_context* c, const rtc_scene* s, const float* rays, uint32_t n,
                                        int32_t depth, int32_t max_depth, int32_t* prim, float* t) {
    return rtc_trace_closest_ex(c, s, rays, n, depth, max_depth, 0, prim, t);
}

extern "C" rtc_status rtc_trace_closest_ex(rtc_context* c, const rtc_scene* s, const float* rays, uint32_t n,
                                           int32_t depth, int32_t max_depth, int32_t flags, int32_t* prim, float* t) {
    if (!c || !s || (n && !rays)) return fail(RTC_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return RTC_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    RtcDeviceScope dev(c->device);
    RTC_CUDA(dev.error());
    float* d_rays = nullptr;
    int32_t* d_prim = nullptr;
    float* d_t = nullptr;
    cudaError_t e = cudaMalloc(&d_rays, (size_t)n * 8 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_prim, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_t, (size_t)n * 4);
    rtc_status r = RTC_OK;
    if (e != cudaSuccess) r = cuda_fail(e, "cudaMalloc(trace)");
    if (r == RTC_OK) {
        e = cudaMemcpyAsync(d_rays, rays, (size_t)n * 8 * sizeof(float), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->d_status, 0, 4, c->stream);
        rtc_render_params vp{};
        vp.flags = flags;
        const DevScene SV = rtc_scene_view(s, &vp);
        auto tfn = SV.num_xnodes ? rtc_launch_trace_closest_x : rtc_launch_trace_closest;
        if (e == cudaSuccess) e = tfn(SV, d_rays, n, depth, max_depth, d_prim, d_t, c->d_status, c->stream);
        if (e == cudaSuccess && prim) e = cudaMemcpyAsync(prim, d_prim, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess && t) e = cudaMemcpyAsync(t, d_t, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "trace_closest");
    }
    cudaFree(d_rays);
    cudaFree(d_prim);
    cudaFree(d_t);
    if (r != RTC_OK) return r;
    return read_status(c);
}

// ---------------------------------------------------------------------------------------------------
// PNG (stored deflate blocks; the reference writes its PNG with stb_image_write, gpu.cu:2110)
// ---------------------------------------------------------------------------------------------------
namespace {
uint32_t crc_table[256];
std::once_flag crc_once;
void crc_init() {
    for (uint32_t n = 0; n < 256; ++n) {
        uint32_t c = n;
        for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xedb88320u ^ (c >> 1) : c >> 1;
        crc_table[n] = c;
    }
}
uint32_t crc32(const uint8_t* p, size_t n, uint32_t c = 0xffffffffu) {
    for (size_t i = 0; i < n; ++i) c = crc_table[(c ^ p[i]) & 0xff] ^ (c >> 8);
    return c;
}
void put32(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back(x >> 24); v.push_back((x >> 16) & 0xff); v.push_back((x >> 8) & 0xff); v.push_back(x & 0xff);
}
void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
    put32(out, (uint32_t)data.size());
    size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data.begin(), data.end());
    uint32_t c = crc32(out.data() + start, out.size() - start) ^ 0xffffffffu;
    put32(out, c);
}
}  // namespace

extern "C" rtc_status rtc_write_png(const char* path, const uint8_t* rgb8, int width, int height) {
    if (!path || !rgb8 || width <= 0 || height <= 0) return fail(RTC_ERR_INVALID_ARGUMENT, "bad PNG arguments");
    std::call_once(crc_once, crc_init);
    std::vector<uint8_t> raw;
    raw.reserve((size_t)height * (width * 3 + 1));
    for (int y = 0; y < height; ++y) {
        raw.push_back(0);   // filter: none
        raw.insert(raw.end(), rgb8 + (size_t)y * width * 3, rgb8 + (size_t)(y + 1) * width * 3);
    }
    std::vector<uint8_t> z;
    z.push_back(0x78);
    z.push_back(0x01);
    uint32_t a = 1, b = 0;
    for (uint8_t x : raw) { a = (a + x) % 65521u; b = (b + a) % 65521u; }
    size_t pos = 0;
    do {
        size_t n = std::min<size_t>(65535, raw.size() - pos);
        bool last = pos + n == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back(n & 0xff); z.push_back(n >> 8);
        z.push_back(~n & 0xff); z.push_back((~n >> 8) & 0xff);
        z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
        pos += n;
    } while (pos < raw.size());
    put32(z, (b << 16) | a);
    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<uint8_t> ihdr;
    put32(ihdr, (uint32_t)width);
    put32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", z);
    chunk(png, "IEND", {});
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(RTC_ERR_IO, std::string("cannot open ") + path);
    size_t w = std::fwrite(png.data(), 1, png.size(), f);
    int cl = std::fclose(f);
    if (w != png.size() || cl != 0) return fail(RTC_ERR_IO, std::string("cannot write ") + path);
    return RTC_OK;
}

extern "C" rtc_status rtc_launchGPU(const rtc_scene_desc* scene, int width, int height, int spp, int max_depth,
                                    int tx, int ty, const char* filepath, int quiet_mode) {
    (void)tx;
    (void)ty;
    if (!scene || !filepath) return fail(RTC_ERR_INVALID_ARGUMENT, "null argument");
    rtc_context* c = nullptr;
    rtc_status r = rtc_context_create(0, &c);
    if (r != RTC_OK) return r;
    rtc_scene* s = nullptr;
    r = rtc_scene_create(c, scene, &s);
    if (r == RTC_OK) {
        rtc_render_params p{width, height, spp, max_depth, 2580u, RTC_MODE_COMPAT, RTC_DRAW_ORDER_DEVICE, 0,
                            RTC_ENGINE_AUTO, 0};
        std::vector<uint8_t> img((size_t)std::max(0, width) * std::max(0, height) * 3);
        if (!quiet_mode) std::printf("[INFO] Rendering %dx%d %d samples > %s\n", width, height, spp, filepath);
        r = rtc_render(c, s, &p, nullptr, img.data());
        if (r == RTC_OK) r = rtc_write_png(filepath, img.data(), width, height);
    }
    std::string keep = g_err;
    rtc_scene_destroy(s);
    rtc_context_destroy(c);
    g_err = keep;
    return r;
}
