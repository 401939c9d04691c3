// ref_harness.cpp - TEST INFRASTRUCTURE ONLY (the oracle).  Never part of the product path.
//
// Compiles the reference's own hot-path classes (flarive/CortexRaytracerCuda core/src/**.cuh) as host
// C++ with g++ (`__device__` expands to nothing when a non-nvcc compiler includes cuda_runtime.h) and
// drives them from an rtc_scene_desc.  Only two things are restated here, both from core/src/gpu.cu:
//   * scene assembly, in the order of load_scene (gpu.cu:481-751): directional lights, spheres,
//     quads, mesh triangles; light list = directional lights (gpu.cu:681-694); camera
//     initialize (gpu.cu:696-725); world = hittable_list(bvh_node(objects, rng(1984))) (gpu.cu:749);
//   * the per-pixel loop of the `render` kernel (gpu.cu:761-790), without quantisation/printf, so the
//     FP32 `pixel_color` sum can be compared.
// Everything else - camera::ray_color, get_ray, every hit/scatter/emitted/pdf/texture function, the
// thrust minstd_rand stream and the reference's BVH - is the reference's code, unmodified.
//
// Built by oracle/Makefile into oracle/_ref/libref_cpu.so (see the recipe there).  Exported C API:
// refh_* below.  The library is loaded by tests/ and by bench.py's cpu_baseline / --impl reference
// legs only.

#include <cuda_runtime.h>
#include <thrust/random.h>

#include "misc/vector3.cuh"
#include "misc/bvh_node.cuh"
#include "primitives/hittable_list.cuh"
#include "textures/texture.cuh"
#include "textures/solid_color_texture.cuh"
#include "textures/checker_texture.cuh"
#include "textures/image_texture.cuh"
#include "materials/diffuse_light.cuh"
#include "materials/lambertian.cuh"
#include "materials/metal.cuh"
#include "materials/dielectric.cuh"
#include "primitives/sphere.cuh"
#include "primitives/quad.cuh"
#include "primitives/triangle.cuh"
#include "primitives/box.cuh"
#include "primitives/translate.cuh"
#include "primitives/rotate.cuh"
#include "primitives/scale.cuh"
#include "lights/light.cuh"
#include "lights/directional_light.cuh"
#include "lights/omni_light.cuh"
#include "lights/spot_light.cuh"
#include "cameras/camera.cuh"
#include "cameras/perspective_camera.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../include/rtc.h"

namespace {

thread_local std::string g_err;

// A reference triangle that also stamps rec.name, so the closest-hit identity can be read back
// (triangle::hit leaves rec.name untouched, core/src/primitives/triangle.cuh:130-185).  Shading is
// unaffected: rec.name is never read by the render path.
class tri_named : public triangle {
public:
    using triangle::triangle;
    bool hit(const ray& r, interval ray_t, hit_record& rec, int depth, int max_depth,
             thrust::default_random_engine& rng) const override {
        if (!triangle::hit(r, ray_t, rec, depth, max_depth, rng)) return false;
        rec.name = m_name;
        return true;
    }
};

// Sky gradient or FP32 environment map behind the camera's background-texture hook
// (camera::ray_color's `if (background_texture)` branch, core/src/cameras/camera.cuh:164-168, which
// calls background_texture->value(u, v, unit_dir)).  The reference's GPU path never sets the hook
// (gpu.cu:729-742), so these backgrounds are parity-unpinned; their formulas are the library's.
class background_tex : public image_texture {
public:
    background_tex(unsigned char* dummy, const rtc_background& bg)
        : image_texture(bitmap_image(dummy, 1, 1, 3)), m_bg(bg) {}
    color value(float, float, const point3& p) const override {
        if (m_bg.kind == RTC_BG_SKY_GRADIENT) {
            float a = 0.5f * (p.y + 1.0f);
            float b = 1.0f - a;
            return color(b * m_bg.color[0] + a * m_bg.top[0], b * m_bg.color[1] + a * m_bg.top[1],
                         b * m_bg.color[2] + a * m_bg.top[2]);
        }
        // equirectangular lookup with get_spherical_uv's convention (uvmapping.cuh:144-158)
        double theta = std::acos((double)-p.y);
        double phi = std::atan2((double)-p.z, (double)p.x) + 3.14159265358979323846;
        double u = phi / (2.0 * 3.14159265358979323846);
        double v = theta / 3.14159265358979323846;
        int W = m_bg.env_width, H = m_bg.env_height;
        int x = (int)(u * W); x = x < 0 ? 0 : (x >= W ? W - 1 : x);
        int y = (int)((1.0 - v) * H); y = y < 0 ? 0 : (y >= H ? H - 1 : y);
        const float* px = m_bg.env_rgb + 3 * ((size_t)y * W + x);
        return color(px[0], px[1], px[2]);
    }
private:
    rtc_background m_bg;
};

// World list that counts closest-hit traversals (for Mrays/s of the reference) and forwards to the
// reference's hittable_list::hit.
class counting_list : public hittable_list {
public:
    explicit counting_list(hittable* h) : hittable_list(h) {}
    bool hit(const ray& r, interval ray_t, hit_record& rec, int depth, int max_depth,
             thrust::default_random_engine& rng) const override {
        ++tl_rays;
        return hittable_list::hit(r, ray_t, rec, depth, max_depth, rng);
    }
    static thread_local uint64_t tl_rays;
};
thread_local uint64_t counting_list::tl_rays = 0;

// Reference-semantics BVH node for scenes where the reference's own O(n^2) exchange sort
// (bvh_node.cuh:94-100) cannot finish: same random-axis median split and the same traversal as
// bvh_node::hit (bvh_node.cuh:110-118), with std::nth_element on the same comparator.  Only the
// topology of ties differs, which changes nothing but the order of equal-t candidates.
class fast_bvh_node : public hittable {
public:
    fast_bvh_node(hittable** objs, size_t start, size_t end, thrust::default_random_engine& rng) {
        thrust::uniform_int_distribution<int> axis_dist(0, 2);
        int axis = axis_dist(rng);
        size_t span = end - start;
        auto cmp = [axis](const hittable* a, const hittable* b) {
            return a->bounding_box().axis(axis).min < b->bounding_box().axis(axis).min;
        };
        if (span == 1) {
            m_left = m_right = objs[start];
        } else if (span == 2) {
            if (cmp(objs[start], objs[start + 1])) { m_left = objs[start]; m_right = objs[start + 1]; }
            else { m_left = objs[start + 1]; m_right = objs[start]; }
        } else {
            size_t mid = start + span / 2;
            std::nth_element(objs + start, objs + mid, objs + end, cmp);
            m_left = new fast_bvh_node(objs, start, mid, rng);
            m_right = new fast_bvh_node(objs, mid, end, rng);
        }
        m_box = aabb(m_left->bounding_box(), m_right->bounding_box());
    }
    bool hit(const ray& r, interval ray_t, hit_record& rec, int depth, int max_depth,
             thrust::default_random_engine& rng) const override {
        if (!m_box.hit(r, ray_t)) return false;
        bool hl = m_left->hit(r, ray_t, rec, depth, max_depth, rng);
        bool hr = m_right->hit(r, interval(ray_t.min, hl ? rec.t : ray_t.max), rec, depth, max_depth, rng);
        return hl || hr;
    }
    float pdf_value(const point3&, const vector3&, int, thrust::default_random_engine&) const override { return 0.0f; }
    vector3 random(const vector3&, thrust::default_random_engine&) const override { return vector3(1, 0, 0); }
    aabb bounding_box() const override { return m_box; }
private:
    hittable* m_left = nullptr;
    hittable* m_right = nullptr;
    aabb m_box;
};

struct ref_scene {
    std::vector<texture*> textures;
    std::vector<material*> materials;
    std::vector<hittable*> objects;     // global primitive order
    std::vector<char> names;            // names[k] is the name storage of primitive k
    hittable_list lights;
    counting_list* world = nullptr;
    rtc_camera cam_desc{};
    rtc_background bg{};
    unsigned char dummy_px[3] = {0, 0, 0};
    background_tex* bg_tex = nullptr;
    std::vector<hittable*> bvh_objects; // the array the BVH constructor sorts in place
};

static vector3 v3(const float* p) { return vector3(p[0], p[1], p[2]); }

// scene_factory::applyTransform (scene_factory.cuh:710-725): translate inside, then rotate, then scale.
static hittable* apply_transform(hittable* h, const rtc_scene_desc* d, uint32_t ref) {
    if (!ref || ref > d->num_transforms) return h;
    const rtc_transform& T = d->transforms[ref - 1];
    if (T.flags & RTC_XF_TRANSLATE) h = new rt::translate(h, v3(T.translate));
    if (T.flags & RTC_XF_ROTATE) h = new rt::rotate(h, v3(T.rotate));
    if (T.flags & RTC_XF_SCALE) h = new rt::scale(h, v3(T.scale));
    return h;
}

static texture* make_texture(ref_scene& s, const rtc_scene_desc* d, int idx, int depth) {
    if (idx < 0 || (uint32_t)idx >= d->num_textures || depth > 4) return nullptr;
    const rtc_texture& t = d->textures[idx];
    switch (t.kind) {
    case RTC_TEX_SOLID:
        return new solid_color_texture(color(t.color[0], t.color[1], t.color[2]));
    case RTC_TEX_CHECKER: {
        texture* even = make_texture(s, d, t.even, depth + 1);
        texture* odd = make_texture(s, d, t.odd, depth + 1);
        if (!even || !odd) return nullptr;
        return new checker_texture(t.scale, even, odd);
    }
    case RTC_TEX_IMAGE: {
        if (t.image < 0 || (uint32_t)t.image >= d->num_images) return nullptr;
        const rtc_image& im = d->images[t.image];
        return new image_texture(bitmap_image(const_cast<unsigned char*>(im.rgb), im.width, im.height, 3));
    }
    }
    return nullptr;
}

// Material construction as scene_factory does it (core/src/scene_factory.cuh: createLambertianMaterial,
// createMetalMaterial, createDielectricMaterial) plus diffuse_light(color, intensity, directional, invisible).
static material* make_material(ref_scene& s, const rtc_scene_desc* d, int idx) {
    if (idx < 0 || (uint32_t)idx >= d->num_materials) return nullptr;
    const rtc_material& m = d->materials[idx];
    switch (m.kind) {
    case RTC_MAT_LAMBERTIAN: {
        texture* t = make_texture(s, d, m.texture, 0);
        return t ? new lambertian(t) : nullptr;
    }
    case RTC_MAT_METAL: {
        if (m.texture < 0 || (uint32_t)m.texture >= d->num_textures) return nullptr;
        const rtc_texture& t = d->textures[m.texture];
        if (t.kind != RTC_TEX_SOLID) return nullptr;  // metal(color, fuzz) only takes a colour
        return new metal(color(t.color[0], t.color[1], t.color[2]), m.fuzz);
    }
    case RTC_MAT_DIELECTRIC:
        return new dielectric(m.ior);
    case RTC_MAT_DIFFUSE_LIGHT: {
        if (m.texture < 0 || (uint32_t)m.texture >= d->num_textures) return nullptr;
        const rtc_texture& t = d->textures[m.texture];
        if (t.kind != RTC_TEX_SOLID) return nullptr;
        return new diffuse_light(color(t.color[0], t.color[1], t.color[2]), m.intensity, m.directional != 0, true);
    }
    }
    return nullptr;
}

}  // namespace

extern "C" {

const char* refh_last_error(void) { return g_err.c_str(); }

// Builds the reference object graph.  bvh_kind: 0 = the reference's bvh_node (O(n^2) build), 1 = the
// harness's fast_bvh_node with the same split rule, -1 = choose by size (reference up to 4096 objects).
void* refh_scene_create(const rtc_scene_desc* d, int bvh_kind) {
    if (!d) { g_err = "null desc"; return nullptr; }
    ref_scene* s = new ref_scene();
    s->cam_desc = d->camera;
    s->bg = d->background;
    uint64_t total = (uint64_t)d->num_omni_lights + d->num_dir_lights + d->num_spot_lights + d->num_spheres + d->num_quads +
                     d->num_boxes;
    for (uint32_t m = 0; m < d->num_meshes; ++m) total += d->meshes[m].num_triangles;
    s->names.assign(total + 1, 0);
    size_t k = 0;
    std::vector<material*> mats(d->num_materials, nullptr);
    for (uint32_t i = 0; i < d->num_materials; ++i) mats[i] = make_material(*s, d, (int)i);
    auto mat_of = [&](int idx) -> material* {
        return (idx >= 0 && (uint32_t)idx < d->num_materials) ? mats[idx] : nullptr;
    };
    // lights in load_scene's order: omni, directional, spot (gpu.cu:504-523)
    for (uint32_t i = 0; i < d->num_omni_lights; ++i, ++k) {
        const rtc_omni_light& L = d->omni_lights[i];
        auto* h = new omni_light(v3(L.position), L.radius, L.intensity, color(L.color[0], L.color[1], L.color[2]),
                                 &s->names[k], L.invisible != 0);
        s->objects.push_back(h);
        s->lights.add(h);
    }
    for (uint32_t i = 0; i < d->num_dir_lights; ++i, ++k) {
        const rtc_dir_light& L = d->dir_lights[i];
        auto* h = new directional_light(v3(L.position), v3(L.u), v3(L.v), L.intensity,
                                        color(L.color[0], L.color[1], L.color[2]), &s->names[k], L.invisible != 0);
        s->objects.push_back(h);
        s->lights.add(h);
    }
    for (uint32_t i = 0; i < d->num_spot_lights; ++i, ++k) {
        const rtc_spot_light& L = d->spot_lights[i];
        auto* h = new spot_light(v3(L.position), v3(L.direction), L.cutoff, L.falloff, L.intensity, L.radius,
                                 color(L.color[0], L.color[1], L.color[2]), &s->names[k], L.invisible != 0);
        s->objects.push_back(h);
        s->lights.add(h);
    }
    for (uint32_t i = 0; i < d->num_spheres; ++i, ++k) {
        const rtc_sphere& S = d->spheres[i];
        material* m = mat_of(S.material);
        if (!m) { g_err = "sphere " + std::to_string(i) + ": bad material"; delete s; return nullptr; }
        s->objects.push_back(apply_transform(new sphere(v3(S.center), S.radius, m, uvmapping(), &s->names[k]), d,
                                             d->sphere_transforms ? d->sphere_transforms[i] : 0));
    }
    for (uint32_t i = 0; i < d->num_quads; ++i, ++k) {
        const rtc_quad& Q = d->quads[i];
        material* m = mat_of(Q.material);
        if (!m) { g_err = "quad " + std::to_string(i) + ": bad material"; delete s; return nullptr; }
        s->objects.push_back(apply_transform(new quad(v3(Q.q), v3(Q.u), v3(Q.v), m, uvmapping(), &s->names[k]), d,
                                             d->quad_transforms ? d->quad_transforms[i] : 0));
    }
    // boxes after the quads (load_scene, gpu.cu:556-565): scene_factory::createBox
    for (uint32_t i = 0; i < d->num_boxes; ++i, ++k) {
        const rtc_box& B = d->boxes[i];
        material* m = mat_of(B.material);
        if (!m) { g_err = "box " + std::to_string(i) + ": bad material"; delete s; return nullptr; }
        s->objects.push_back(apply_transform(new box(v3(B.center), v3(B.size), m, uvmapping(), &s->names[k]), d,
                                             B.transform));
    }
    for (uint32_t mi = 0; mi < d->num_meshes; ++mi) {
        const rtc_mesh& M = d->meshes[mi];
        material* m = mat_of(M.material);
        if (!m) { g_err = "mesh " + std::to_string(mi) + ": bad material"; delete s; return nullptr; }
        for (uint32_t f = 0; f < M.num_triangles; ++f, ++k) {
            uint32_t ia = M.indices[3 * f], ib = M.indices[3 * f + 1], ic = M.indices[3 * f + 2];
            if (ia >= M.num_vertices || ib >= M.num_vertices || ic >= M.num_vertices) {
                g_err = "mesh index out of range"; delete s; return nullptr;
            }
            vector3 a = v3(M.vertices + 3 * ia), b = v3(M.vertices + 3 * ib), c = v3(M.vertices + 3 * ic);
            tri_named* t;
            if (M.smooth && M.normals) {
                vector2 ua(0), ub(0), uc(0);
                if (M.uvs) {
                    ua = vector2(M.uvs[2 * ia], M.uvs[2 * ia + 1]);
                    ub = vector2(M.uvs[2 * ib], M.uvs[2 * ib + 1]);
                    uc = vector2(M.uvs[2 * ic], M.uvs[2 * ic + 1]);
                }
                // the full constructor is the one mesh_loader uses (mesh_loader.cuh:395-401)
                t = new tri_named(a, b, c, v3(M.normals + 3 * ia), v3(M.normals + 3 * ib), v3(M.normals + 3 * ic),
                                  ua, ub, uc, vector3(), vector3(), vector3(), vector3(), vector3(), vector3(),
                                  true, m, &s->names[k]);
            } else {
                t = new tri_named(a, b, c, m, &s->names[k]);
            }
            t->setName(&s->names[k]);
            s->objects.push_back(apply_transform(t, d, d->mesh_transforms ? d->mesh_transforms[mi] : 0));
        }
    }
    if (s->objects.empty()) { g_err = "empty scene"; delete s; return nullptr; }
    // world = hittable_list(new bvh_node(objects, 0, n, rng(1984)))  (gpu.cu:749, seed gpu.cu:2068)
    s->bvh_objects = s->objects;
    thrust::minstd_rand rng(1984);
    bool use_ref = bvh_kind == 0 || (bvh_kind < 0 && s->objects.size() <= 4096);
    hittable* root;
    if (use_ref)
        root = new bvh_node(s->bvh_objects.data(), 0, (int)s->bvh_objects.size(), rng);
    else
        root = new fast_bvh_node(s->bvh_objects.data(), 0, s->bvh_objects.size(), rng);
    s->world = new counting_list(root);
    if (d->background.kind != RTC_BG_CONSTANT) s->bg_tex = new background_tex(s->dummy_px, d->background);
    return s;
}

void refh_scene_destroy(void* p) {
    // The reference never frees its device-heap object graph either (gpu.cu:2118-2123); the harness
    // releases only what it allocated around it.
    delete static_cast<ref_scene*>(p);
}

int refh_num_objects(void* p) { return p ? (int)static_cast<ref_scene*>(p)->objects.size() : -1; }

// Renders the listed pixels.  out_rgba[4*k..] = the reference's FP32 pixel_color sum (RGBA) of pixel
// pix[k] (index j*width + i, j from the bottom); out_rays (may be NULL) = closest-hit traversals.
int refh_render_pixels(void* p, const rtc_render_params* prm, const int64_t* pix, int64_t n,
                       float* out_rgba, uint64_t* out_rays, int threads) {
    ref_scene* s = static_cast<ref_scene*>(p);
    if (!s || !prm || (!pix && n > 0) || !out_rgba) { g_err = "bad argument"; return 1; }
    const int width = prm->width, height = prm->height, spp = prm->spp, max_depth = prm->max_depth;
    const int sqrt_spp = (int)std::sqrt((float)spp);   // gpu.cu:1989
    perspective_camera cam;
    cam.vfov = s->cam_desc.vfov;
    cam.initialize(v3(s->cam_desc.look_from), v3(s->cam_desc.look_at), v3(s->cam_desc.up), width,
                   s->cam_desc.aspect, s->cam_desc.vfov, s->cam_desc.aperture, s->cam_desc.focus, 0.0f, 0.0f,
                   1.0f, sqrt_spp);
    cam.samples_per_pixel = spp;
    cam.max_depth = max_depth;
    cam.background_color = color(s->bg.color[0], s->bg.color[1], s->bg.color[2]);
    if (s->bg_tex) { cam.background_texture = s->bg_tex; cam.background_iskybox = true; }

    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int64_t> next{0};
    std::atomic<uint64_t> rays{0};
    const int64_t chunk = 16;
    auto worker = [&]() {
        counting_list::tl_rays = 0;
        for (;;) {
            int64_t b = next.fetch_add(chunk);
            if (b >= n) break;
            int64_t e = std::min(n, b + chunk);
            for (int64_t q = b; q < e; ++q) {
                int64_t pixel_index = pix[q];
                int i = (int)(pixel_index % width), j = (int)(pixel_index / width);
                // render kernel body (gpu.cu:769-790)
                thrust::minstd_rand rng(prm->seed + (uint32_t)pixel_index);
                thrust::uniform_real_distribution<float> uniform_dist(0.0f, 1.0f);
                color pixel_color(0, 0, 0);
                for (int s_j = 0; s_j < sqrt_spp; ++s_j) {
                    for (int s_i = 0; s_i < sqrt_spp; ++s_i) {
                        float uniform_random = uniform_dist(rng);
                        float u = (i + (s_i + uniform_random) / sqrt_spp) / float(width);
                        float v = (j + (s_j + uniform_random) / sqrt_spp) / float(height);
                        ray r = cam.get_ray(u, v, s_i, s_j, nullptr, rng);
                        pixel_color += cam.ray_color(r, i, j, max_depth, max_depth, *s->world, s->lights, rng);
                    }
                }
                out_rgba[4 * q + 0] = pixel_color.r();
                out_rgba[4 * q + 1] = pixel_color.g();
                out_rgba[4 * q + 2] = pixel_color.b();
                out_rgba[4 * q + 3] = pixel_color.a();
            }
        }
        rays.fetch_add(counting_list::tl_rays);
    };
    if (threads == 1) {
        worker();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
    }
    if (out_rays) *out_rays = rays.load();
    return 0;
}

// Closest-hit identity on arbitrary rays through the reference's world.hit.  rays: n x 8 floats
// (ox, oy, oz, tmin, dx, dy, dz, tmax).  prim[k] = global primitive id or -1.
int refh_trace_closest(void* p, const float* rays, int64_t n, int depth, int max_depth, int32_t* prim,
                       float* tout) {
    ref_scene* s = static_cast<ref_scene*>(p);
    if (!s || !rays) { g_err = "bad argument"; return 1; }
    thrust::minstd_rand rng(1);
    for (int64_t k = 0; k < n; ++k) {
        const float* R = rays + 8 * k;
        ray r(point3(R[0], R[1], R[2]), vector3(R[4], R[5], R[6]), 0.0f);
        hit_record rec;
        bool h = s->world->hit(r, interval(R[3], R[7]), rec, depth, max_depth, rng);
        int32_t id = -1;
        if (h && rec.name) id = (int32_t)(rec.name - s->names.data());
        if (prim) prim[k] = id;
        if (tout) tout[k] = h ? rec.t : INFINITY;
    }
    return 0;
}

// thrust::minstd_rand(seed) -> uniform_real_distribution<float>(0,1), n draws (the T0 known-answer test).
int refh_rng_draws(uint32_t seed, int64_t n, float* out) {
    thrust::minstd_rand rng(seed);
    thrust::uniform_real_distribution<float> dist(0.0f, 1.0f);
    for (int64_t k = 0; k < n; ++k) out[k] = dist(rng);
    return 0;
}

// get_int (gpu_randomizer.cuh:29-35) for n draws of [lo, hi].
int refh_get_int(uint32_t seed, int lo, int hi, int64_t n, int32_t* out) {
    thrust::minstd_rand rng(seed);
    for (int64_t k = 0; k < n; ++k) out[k] = get_int(rng, lo, hi);
    return 0;
}

// The reference's multi-draw helpers as this (g++) build evaluates them; 3 floats per call:
// which = 0 random_in_unit_disk, 1 random_in_unit_sphere, 2 random_cosine_direction,
//         3 directional_light::random for light (0,0,0), u=(1,0,0), v=(0,1,0) seen from the origin,
//         4 omni_light::random for a light at (0.3,-0.2,0.1), radius 0.5, seen from (1.3,0.7,-2.1).
int refh_sampler_draws(int which, uint32_t seed, int64_t n, float* out) {
    thrust::minstd_rand rng(seed);
    directional_light L(point3(0, 0, 0), vector3(1, 0, 0), vector3(0, 1, 0), 1.0f, color(1, 1, 1));
    for (int64_t k = 0; k < n; ++k) {
        vector3 p;
        switch (which) {
        case 0: p = random_in_unit_disk(rng); break;
        case 1: p = random_in_unit_sphere(rng); break;
        case 2: p = random_cosine_direction(rng); break;
        case 3: p = L.random(point3(0, 0, 0), rng); break;
        case 4: {   // omni_light::random for a light at (0.3, -0.2, 0.1), radius 0.5, seen from (1.3, 0.7, -2.1)
            static omni_light O(point3(0.3f, -0.2f, 0.1f), 0.5f, 1.0f, color(1, 1, 1));
            p = O.random(point3(1.3f, 0.7f, -2.1f), rng);
        } break;
        case 5: p = random_to_sphere(rng, 0.5f, 4.0f); break;
        default: g_err = "bad sampler"; return 1;
        }
        out[3 * k] = p.x; out[3 * k + 1] = p.y; out[3 * k + 2] = p.z;
    }
    return 0;
}

// Camera rays of pixel (i, j) for its sqrt_spp^2 samples, rays: n_samples x 7 floats (origin, dir, time).
int refh_camera_rays(void* p, const rtc_render_params* prm, int i, int j, float* out) {
    ref_scene* s = static_cast<ref_scene*>(p);
    if (!s || !prm || !out) return 1;
    const int sqrt_spp = (int)std::sqrt((float)prm->spp);
    perspective_camera cam;
    cam.initialize(v3(s->cam_desc.look_from), v3(s->cam_desc.look_at), v3(s->cam_desc.up), prm->width,
                   s->cam_desc.aspect, s->cam_desc.vfov, s->cam_desc.aperture, s->cam_desc.focus, 0.0f, 0.0f,
                   1.0f, sqrt_spp);
    thrust::minstd_rand rng(prm->seed + (uint32_t)(j * prm->width + i));
    thrust::uniform_real_distribution<float> uniform_dist(0.0f, 1.0f);
    int q = 0;
    for (int s_j = 0; s_j < sqrt_spp; ++s_j)
        for (int s_i = 0; s_i < sqrt_spp; ++s_i, ++q) {
            float uniform_random = uniform_dist(rng);
            float u = (i + (s_i + uniform_random) / sqrt_spp) / float(prm->width);
            float v = (j + (s_j + uniform_random) / sqrt_spp) / float(prm->height);
            ray r = cam.get_ray(u, v, s_i, s_j, nullptr, rng);
            float* o = out + 7 * q;
            o[0] = r.origin().x; o[1] = r.origin().y; o[2] = r.origin().z;
            o[3] = r.direction().x; o[4] = r.direction().y; o[5] = r.direction().z;
            o[6] = r.time();
        }
    return 0;
}

}  // extern "C"
