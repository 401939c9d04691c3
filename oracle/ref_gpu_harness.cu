// ref_gpu_harness.cu - TEST INFRASTRUCTURE ONLY (the oracle, GPU build).  Never part of the product.
//
// The reference's own hot-path classes (flarive/CortexRaytracerCuda core/src/**.cuh) compiled by nvcc
// for sm_100a, exactly as the reference's gpu.cu compiles them: the object graph is built on the
// device by one thread with device `new` (as load_scene does, core/src/gpu.cu:481-751), the BVH is
// the reference's bvh_node with thrust::minstd_rand(1984) (gpu.cu:749, 2068), and a render kernel
// restates the `render` kernel body (gpu.cu:761-790) but stores the FP32 pixel_color sum instead of
// quantising and printf-ing it.  This is the oracle for the reference's *device* RNG consumption
// order, which differs from a g++ build (see refg_sampler_draws).
//
// Built by oracle/Makefile into _ref/libref_gpu.so.  Exported C API: refg_* below.

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
#include "lights/light.cuh"
#include "lights/directional_light.cuh"
#include "cameras/camera.cuh"
#include "cameras/perspective_camera.cuh"

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../include/rtc.h"

namespace {

thread_local std::string g_err;

// device copies of the description arrays
struct DDesc {
    rtc_texture* tex; int ntex;
    rtc_material* mat; int nmat;
    rtc_dir_light* lights; int nlights;
    rtc_sphere* sph; int nsph;
    rtc_quad* quads; int nquads;
    float* verts; uint32_t* idx; int* tri_mat; int ntri;   // flattened triangles (flat normals only)
    unsigned char** img_data; int* img_w; int* img_h; int nimg;
    rtc_camera cam;
    rtc_background bg;
    const float* env;          // environment map (RTC_BG_ENV_MAP), device copy
    unsigned char* dummy_px;   // the 1x1 bitmap the background texture's base class holds
};

struct DWorld {
    hittable_list* world;
    hittable_list* lights;
    hittable** objects;
    int n;
    char* names;   // names[k] = name storage of primitive k
    image_texture* bg_tex;   // sky gradient / environment map behind the camera's background hook, or null
};

// Sky gradient or FP32 environment map behind the camera's background-texture hook
// (camera::ray_color's `if (background_texture)` branch, core/src/cameras/camera.cuh:164-168, which calls
// background_texture->value(u, v, unit_dir)); the device twin of ref_harness.cpp's background_tex.  The
// reference's GPU path never sets the hook (gpu.cu:729-742), so these backgrounds are parity-unpinned and
// their formulas are the library's; the hook, the loop around it and everything it multiplies are the
// reference's own code.
class refg_background : public image_texture {
public:
    __host__ __device__ refg_background(unsigned char* dummy, const rtc_background& bg, const float* env)
        : image_texture(bitmap_image(dummy, 1, 1, 3)), m_bg(bg), m_env(env) {}
    __host__ __device__ color value(float, float, const point3& p) const override {
        if (m_bg.kind == RTC_BG_SKY_GRADIENT) {
            float a = 0.5f * (p.y + 1.0f);
            float b = 1.0f - a;
            return color(b * m_bg.color[0] + a * m_bg.top[0], b * m_bg.color[1] + a * m_bg.top[1],
                         b * m_bg.color[2] + a * m_bg.top[2]);
        }
        // equirectangular lookup with get_spherical_uv's convention (uvmapping.cuh:144-158)
        double theta = acos((double)-p.y);
        double phi = atan2((double)-p.z, (double)p.x) + 3.14159265358979323846;
        double u = phi / (2.0 * 3.14159265358979323846);
        double v = theta / 3.14159265358979323846;
        int W = m_bg.env_width, H = m_bg.env_height;
        int x = (int)(u * W); x = x < 0 ? 0 : (x >= W ? W - 1 : x);
        int y = (int)((1.0 - v) * H); y = y < 0 ? 0 : (y >= H ? H - 1 : y);
        const float* px = m_env + 3 * ((size_t)y * W + x);
        return color(px[0], px[1], px[2]);
    }
private:
    rtc_background m_bg;
    const float* m_env;
};

__device__ vector3 dv3(const float* p) { return vector3(p[0], p[1], p[2]); }

__device__ texture* dmake_tex(const DDesc& d, int idx, int depth) {
    if (idx < 0 || idx >= d.ntex || depth > 4) return nullptr;
    const rtc_texture& t = d.tex[idx];
    if (t.kind == RTC_TEX_SOLID) return new solid_color_texture(color(t.color[0], t.color[1], t.color[2]));
    if (t.kind == RTC_TEX_CHECKER) {
        texture* e = dmake_tex(d, t.even, depth + 1);
        texture* o = dmake_tex(d, t.odd, depth + 1);
        if (!e || !o) return nullptr;
        return new checker_texture(t.scale, e, o);
    }
    if (t.kind == RTC_TEX_IMAGE && t.image >= 0 && t.image < d.nimg)
        return new image_texture(bitmap_image(d.img_data[t.image], d.img_w[t.image], d.img_h[t.image], 3));
    return nullptr;
}

__device__ material* dmake_mat(const DDesc& d, int idx) {
    if (idx < 0 || idx >= d.nmat) return nullptr;
    const rtc_material& m = d.mat[idx];
    if (m.kind == RTC_MAT_LAMBERTIAN) {
        texture* t = dmake_tex(d, m.texture, 0);
        return t ? new lambertian(t) : nullptr;
    }
    if (m.kind == RTC_MAT_DIELECTRIC) return new dielectric(m.ior);
    if (m.texture < 0 || m.texture >= d.ntex || d.tex[m.texture].kind != RTC_TEX_SOLID) return nullptr;
    const rtc_texture& t = d.tex[m.texture];
    color c(t.color[0], t.color[1], t.color[2]);
    if (m.kind == RTC_MAT_METAL) return new metal(c, m.fuzz);
    if (m.kind == RTC_MAT_DIFFUSE_LIGHT) return new diffuse_light(c, m.intensity, m.directional != 0, true);
    return nullptr;
}

// the reference's load_scene object order (gpu.cu:504-635) and light extraction (gpu.cu:681-694)
__global__ void refg_load_scene(DDesc d, DWorld* out, int* ok) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    *ok = 0;
    int n = d.nlights + d.nsph + d.nquads + d.ntri;
    hittable** objs = new hittable*[n > 0 ? n : 1];
    char* names = new char[n + 1];
    material** mats = new material*[d.nmat > 0 ? d.nmat : 1];
    for (int i = 0; i < d.nmat; ++i) mats[i] = dmake_mat(d, i);
    hittable_list* lights = new hittable_list();
    int k = 0;
    for (int i = 0; i < d.nlights; ++i, ++k) {
        const rtc_dir_light& L = d.lights[i];
        directional_light* h = new directional_light(dv3(L.position), dv3(L.u), dv3(L.v), L.intensity,
                                                     color(L.color[0], L.color[1], L.color[2]), &names[k], L.invisible != 0);
        objs[k] = h;
        lights->add(h);
    }
    for (int i = 0; i < d.nsph; ++i, ++k) {
        material* m = (d.sph[i].material >= 0 && d.sph[i].material < d.nmat) ? mats[d.sph[i].material] : nullptr;
        if (!m) return;
        objs[k] = new sphere(dv3(d.sph[i].center), d.sph[i].radius, m, uvmapping(), &names[k]);
    }
    for (int i = 0; i < d.nquads; ++i, ++k) {
        material* m = (d.quads[i].material >= 0 && d.quads[i].material < d.nmat) ? mats[d.quads[i].material] : nullptr;
        if (!m) return;
        objs[k] = new quad(dv3(d.quads[i].q), dv3(d.quads[i].u), dv3(d.quads[i].v), m, uvmapping(), &names[k]);
    }
    for (int f = 0; f < d.ntri; ++f, ++k) {
        material* m = (d.tri_mat[f] >= 0 && d.tri_mat[f] < d.nmat) ? mats[d.tri_mat[f]] : nullptr;
        if (!m) return;
        triangle* t = new triangle(dv3(d.verts + 9 * f), dv3(d.verts + 9 * f + 3), dv3(d.verts + 9 * f + 6), m, &names[k]);
        t->setName(&names[k]);
        objs[k] = t;
    }
    thrust::minstd_rand rng(1984);
    out->world = new hittable_list(new bvh_node(objs, 0, n, rng));
    out->lights = lights;
    out->objects = objs;
    out->n = n;
    out->names = names;
    out->bg_tex = d.bg.kind != RTC_BG_CONSTANT ? new refg_background(d.dummy_px, d.bg, d.env) : nullptr;
    *ok = 1;
}

// One pixel of the `render` kernel (gpu.cu:767-790): its FP32 pixel_color sum, before
// prepare_pixel_color.  The camera is the reference's perspective_camera, initialised as load_scene does.
__device__ color refg_pixel(DWorld* w, const rtc_camera& cd, const rtc_background& bg, const rtc_render_params& p,
                            int sqrt_spp, int64_t pixel_index) {
    perspective_camera cam;
    cam.vfov = cd.vfov;
    cam.initialize(dv3(cd.look_from), dv3(cd.look_at), dv3(cd.up), p.width, cd.aspect, cd.vfov, cd.aperture, cd.focus,
                   0.0f, 0.0f, 1.0f, sqrt_spp);
    cam.samples_per_pixel = p.spp;
    cam.max_depth = p.max_depth;
    cam.background_color = color(bg.color[0], bg.color[1], bg.color[2]);
    if (w->bg_tex) { cam.background_texture = w->bg_tex; cam.background_iskybox = true; }
    int i = (int)(pixel_index % p.width), j = (int)(pixel_index / p.width);
    thrust::minstd_rand rng(p.seed + (uint32_t)pixel_index);
    thrust::uniform_real_distribution<float> uniform_dist(0.0f, 1.0f);
    color pixel_color(0, 0, 0);
    for (int s_j = 0; s_j < sqrt_spp; ++s_j) {
        for (int s_i = 0; s_i < sqrt_spp; ++s_i) {
            float uniform_random = uniform_dist(rng);
            float u = (i + (s_i + uniform_random) / sqrt_spp) / float(p.width);
            float v = (j + (s_j + uniform_random) / sqrt_spp) / float(p.height);
            ray r = cam.get_ray(u, v, s_i, s_j, nullptr, rng);
            pixel_color += cam.ray_color(r, i, j, p.max_depth, p.max_depth, *w->world, *w->lights, rng);
        }
    }
    return pixel_color;
}

// the render kernel body over a list of pixels (gpu.cu:761-790), without quantisation / printf
__global__ void refg_render(DWorld* w, rtc_camera cd, rtc_background bg, rtc_render_params p, int sqrt_spp,
                            const int64_t* pix, int64_t n, float* out) {
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const color pixel_color = refg_pixel(w, cd, bg, p, sqrt_spp, pix[q]);
    out[4 * q + 0] = pixel_color.r();
    out[4 * q + 1] = pixel_color.g();
    out[4 * q + 2] = pixel_color.b();
    out[4 * q + 3] = pixel_color.a();
}

// The whole frame in the reference's launch shape (gpu.cu:2072-2080): (W/16+1, H/16+1) blocks of 16x16
// threads, thread (i, j) renders pixel j*W+i (gpu.cu:763-767).  Stores the FP32 sum where the reference
// stores the quantised colour and prints it (the per-pixel printf is left out).
__global__ void refg_render_frame(DWorld* w, rtc_camera cd, rtc_background bg, rtc_render_params p, int sqrt_spp,
                                  float* out) {
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    int j = threadIdx.y + blockIdx.y * blockDim.y;
    if ((i >= p.width) || (j >= p.height)) return;
    const int64_t q = (int64_t)j * p.width + i;
    const color pixel_color = refg_pixel(w, cd, bg, p, sqrt_spp, q);
    out[4 * q + 0] = pixel_color.r();
    out[4 * q + 1] = pixel_color.g();
    out[4 * q + 2] = pixel_color.b();
    out[4 * q + 3] = pixel_color.a();
}

__global__ void refg_trace(DWorld* w, const float* rays, int64_t n, int depth, int max_depth, int32_t* prim, float* tout) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float* R = rays + 8 * k;
    thrust::minstd_rand rng(1);
    ray r(point3(R[0], R[1], R[2]), vector3(R[4], R[5], R[6]), 0.0f);
    hit_record rec;
    bool h = w->world->hit(r, interval(R[3], R[7]), rec, depth, max_depth, rng);
    prim[k] = (h && rec.name) ? (int32_t)(rec.name - w->names) : -1;
    tout[k] = h ? rec.t : INFINITY;
}

__global__ void refg_camera(rtc_camera cd, rtc_render_params p, int sqrt_spp, int i, int j, float* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    perspective_camera cam;
    cam.initialize(dv3(cd.look_from), dv3(cd.look_at), dv3(cd.up), p.width, cd.aspect, cd.vfov, cd.aperture, cd.focus,
                   0.0f, 0.0f, 1.0f, sqrt_spp);
    thrust::minstd_rand rng(p.seed + (uint32_t)(j * p.width + i));
    thrust::uniform_real_distribution<float> uniform_dist(0.0f, 1.0f);
    int q = 0;
    for (int s_j = 0; s_j < sqrt_spp; ++s_j)
        for (int s_i = 0; s_i < sqrt_spp; ++s_i, ++q) {
            float uniform_random = uniform_dist(rng);
            float u = (i + (s_i + uniform_random) / sqrt_spp) / float(p.width);
            float v = (j + (s_j + uniform_random) / sqrt_spp) / float(p.height);
            ray r = cam.get_ray(u, v, s_i, s_j, nullptr, rng);
            float* o = out + 7 * q;
            o[0] = r.origin().x; o[1] = r.origin().y; o[2] = r.origin().z;
            o[3] = r.direction().x; o[4] = r.direction().y; o[5] = r.direction().z;
            o[6] = r.time();
        }
}

__global__ void refg_samplers(int which, uint32_t seed, int64_t n, float* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    thrust::minstd_rand rng(seed);
    directional_light L(point3(0, 0, 0), vector3(1, 0, 0), vector3(0, 1, 0), 1.0f, color(1, 1, 1));
    for (int64_t k = 0; k < n; ++k) {
        vector3 p;
        if (which == 0) p = random_in_unit_disk(rng);
        else if (which == 1) p = random_in_unit_sphere(rng);
        else if (which == 2) p = random_cosine_direction(rng);
        else p = L.random(point3(0, 0, 0), rng);
        out[3 * k] = p.x; out[3 * k + 1] = p.y; out[3 * k + 2] = p.z;
    }
}

template <class T>
T* upload(const T* src, size_t n, std::vector<void*>& allocs) {
    if (!n) return nullptr;
    T* d = nullptr;
    if (cudaMalloc(&d, n * sizeof(T)) != cudaSuccess) return nullptr;
    allocs.push_back(d);
    cudaMemcpy(d, src, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

struct GpuScene {
    DWorld* d_world = nullptr;
    std::vector<void*> allocs;
    rtc_camera cam;
    rtc_background bg;
};

bool check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

}  // namespace

extern "C" {

const char* refg_last_error(void) { return g_err.c_str(); }

// Device limits as the reference's setupCuda sets them (gpu.cu:805-855), minus the printf FIFO.
int refg_setup(void) {
    if (!check(cudaDeviceSetLimit(cudaLimitStackSize, 4096), "stack limit")) return 1;
    if (!check(cudaDeviceSetLimit(cudaLimitMallocHeapSize, size_t(1) << 30), "heap limit")) return 1;
    return 0;
}

void* refg_scene_create(const rtc_scene_desc* d) {
    if (!d) return nullptr;
    GpuScene* s = new GpuScene();
    DDesc dd{};
    dd.bg = d->background;
    if (d->background.kind == RTC_BG_ENV_MAP)
        dd.env = upload(d->background.env_rgb, (size_t)3 * d->background.env_width * d->background.env_height, s->allocs);
    const unsigned char px[3] = {0, 0, 0};
    dd.dummy_px = upload(px, 3, s->allocs);
    dd.tex = upload(d->textures, d->num_textures, s->allocs); dd.ntex = d->num_textures;
    dd.mat = upload(d->materials, d->num_materials, s->allocs); dd.nmat = d->num_materials;
    dd.lights = upload(d->dir_lights, d->num_dir_lights, s->allocs); dd.nlights = d->num_dir_lights;
    dd.sph = upload(d->spheres, d->num_spheres, s->allocs); dd.nsph = d->num_spheres;
    dd.quads = upload(d->quads, d->num_quads, s->allocs); dd.nquads = d->num_quads;
    std::vector<float> verts;
    std::vector<int> tmat;
    for (uint32_t m = 0; m < d->num_meshes; ++m) {
        const rtc_mesh& M = d->meshes[m];
        if (M.smooth) { g_err = "smooth meshes are not supported by the GPU harness"; delete s; return nullptr; }
        for (uint32_t f = 0; f < M.num_triangles; ++f) {
            for (int c = 0; c < 3; ++c) {
                uint32_t vi = M.indices[3 * f + c];
                verts.insert(verts.end(), M.vertices + 3 * vi, M.vertices + 3 * vi + 3);
            }
            tmat.push_back(M.material);
        }
    }
    dd.verts = upload(verts.data(), verts.size(), s->allocs);
    dd.tri_mat = upload(tmat.data(), tmat.size(), s->allocs);
    dd.ntri = (int)tmat.size();
    std::vector<unsigned char*> dimg;
    std::vector<int> iw, ih;
    for (uint32_t i = 0; i < d->num_images; ++i) {
        const rtc_image& im = d->images[i];
        dimg.push_back(upload(im.rgb, (size_t)im.width * im.height * 3, s->allocs));
        iw.push_back(im.width);
        ih.push_back(im.height);
    }
    dd.img_data = upload(dimg.data(), dimg.size(), s->allocs);
    dd.img_w = upload(iw.data(), iw.size(), s->allocs);
    dd.img_h = upload(ih.data(), ih.size(), s->allocs);
    dd.nimg = (int)dimg.size();
    s->cam = d->camera;
    s->bg = d->background;
    DWorld* dw = nullptr;
    int* dok = nullptr;
    if (!check(cudaMalloc(&dw, sizeof(DWorld)), "malloc world") || !check(cudaMalloc(&dok, sizeof(int)), "malloc ok")) {
        delete s; return nullptr;
    }
    s->allocs.push_back(dw);
    s->allocs.push_back(dok);
    s->d_world = dw;
    refg_load_scene<<<1, 1>>>(dd, dw, dok);
    int ok = 0;
    if (!check(cudaDeviceSynchronize(), "load_scene") || !check(cudaMemcpy(&ok, dok, sizeof(int), cudaMemcpyDeviceToHost), "ok")) {
        delete s; return nullptr;
    }
    if (!ok) { g_err = "device scene construction failed (bad material reference)"; delete s; return nullptr; }
    return s;
}

void refg_scene_destroy(void* p) {
    GpuScene* s = static_cast<GpuScene*>(p);
    if (!s) return;
    for (void* a : s->allocs) cudaFree(a);   // the device-heap object graph stays until context teardown,
    delete s;                                // as in the reference (gpu.cu:2118-2123)
}

int refg_render_pixels(void* p, const rtc_render_params* prm, const int64_t* pix, int64_t n, float* out_rgba) {
    GpuScene* s = static_cast<GpuScene*>(p);
    if (!s || !prm || n <= 0) { g_err = "bad argument"; return 1; }
    int sqrt_spp = (int)std::sqrt((double)prm->spp);
    int64_t* dpix = nullptr;
    float* dout = nullptr;
    if (!check(cudaMalloc(&dpix, n * sizeof(int64_t)), "malloc") || !check(cudaMalloc(&dout, n * 16), "malloc")) return 1;
    cudaMemcpy(dpix, pix, n * sizeof(int64_t), cudaMemcpyHostToDevice);
    refg_render<<<(unsigned)((n + 63) / 64), 64>>>(s->d_world, s->cam, s->bg, *prm, sqrt_spp, dpix, n, dout);
    bool ok = check(cudaDeviceSynchronize(), "refg_render");
    if (ok) ok = check(cudaMemcpy(out_rgba, dout, n * 16, cudaMemcpyDeviceToHost), "copy");
    cudaFree(dpix);
    cudaFree(dout);
    return ok ? 0 : 1;
}

// Renders the whole frame with refg_render_frame; `ms` receives the kernel's CUDA-event time (the
// device-heap object graph is already built; allocation and copies are outside the events).
// `out_rgba` (may be null) receives width*height float4 sums in frame-buffer order.
int refg_render_frame_timed(void* p, const rtc_render_params* prm, float* out_rgba, float* ms) {
    GpuScene* s = static_cast<GpuScene*>(p);
    if (!s || !prm || !ms || prm->width <= 0 || prm->height <= 0) { g_err = "bad argument"; return 1; }
    const int sqrt_spp = (int)std::sqrt((double)prm->spp);
    const size_t npix = (size_t)prm->width * prm->height;
    float* dout = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!check(cudaMalloc(&dout, npix * 16), "malloc")) return 1;
    bool ok = check(cudaEventCreate(&e0), "event") && check(cudaEventCreate(&e1), "event");
    if (ok) {
        const int tx = 16, ty = 16;   // gpu_cuda_renderer passes tx = ty = 16 (renderers/gpu_cuda_renderer.h:23-27)
        dim3 blocks(prm->width / tx + 1, prm->height / ty + 1), threads(tx, ty);
        cudaEventRecord(e0, 0);
        refg_render_frame<<<blocks, threads>>>(s->d_world, s->cam, s->bg, *prm, sqrt_spp, dout);
        cudaEventRecord(e1, 0);
        ok = check(cudaGetLastError(), "refg_render_frame") && check(cudaDeviceSynchronize(), "refg_render_frame") &&
             check(cudaEventElapsedTime(ms, e0, e1), "elapsed");
    }
    if (ok && out_rgba) ok = check(cudaMemcpy(out_rgba, dout, npix * 16, cudaMemcpyDeviceToHost), "copy");
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(dout);
    return ok ? 0 : 1;
}

int refg_trace_closest(void* p, const float* rays, int64_t n, int depth, int max_depth, int32_t* prim, float* tout) {
    GpuScene* s = static_cast<GpuScene*>(p);
    if (!s || n <= 0) { g_err = "bad argument"; return 1; }
    float* dr = nullptr; int32_t* dp = nullptr; float* dt = nullptr;
    if (!check(cudaMalloc(&dr, n * 32), "malloc") || !check(cudaMalloc(&dp, n * 4), "malloc") || !check(cudaMalloc(&dt, n * 4), "malloc"))
        return 1;
    cudaMemcpy(dr, rays, n * 32, cudaMemcpyHostToDevice);
    refg_trace<<<(unsigned)((n + 127) / 128), 128>>>(s->d_world, dr, n, depth, max_depth, dp, dt);
    bool ok = check(cudaDeviceSynchronize(), "refg_trace");
    if (ok) ok = check(cudaMemcpy(prim, dp, n * 4, cudaMemcpyDeviceToHost), "copy") &&
                 check(cudaMemcpy(tout, dt, n * 4, cudaMemcpyDeviceToHost), "copy");
    cudaFree(dr); cudaFree(dp); cudaFree(dt);
    return ok ? 0 : 1;
}

int refg_camera_rays(void* p, const rtc_render_params* prm, int i, int j, float* out) {
    GpuScene* s = static_cast<GpuScene*>(p);
    if (!s || !prm || !out) return 1;
    int sq = (int)std::sqrt((double)prm->spp);
    float* d = nullptr;
    if (!check(cudaMalloc(&d, (size_t)sq * sq * 28), "malloc")) return 1;
    refg_camera<<<1, 1>>>(s->cam, *prm, sq, i, j, d);
    bool ok = check(cudaDeviceSynchronize(), "refg_camera") && check(cudaMemcpy(out, d, (size_t)sq * sq * 28, cudaMemcpyDeviceToHost), "copy");
    cudaFree(d);
    return ok ? 0 : 1;
}

int refg_sampler_draws(int which, uint32_t seed, int64_t n, float* out) {
    float* d = nullptr;
    if (!check(cudaMalloc(&d, n * 12), "malloc")) return 1;
    refg_samplers<<<1, 1>>>(which, seed, n, d);
    bool ok = check(cudaDeviceSynchronize(), "refg_samplers") && check(cudaMemcpy(out, d, n * 12, cudaMemcpyDeviceToHost), "copy");
    cudaFree(d);
    return ok ? 0 : 1;
}

}  // extern "C"
