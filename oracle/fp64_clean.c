/* fp64_clean.c - TEST INFRASTRUCTURE ONLY (the converged-image oracle).  Never part of the product path.
 *
 * A double-precision restatement of the clean-mode estimator, for converged-image comparisons
 * (RMSE against the FP32 kernels at high spp).  It evaluates the same estimator as the clean kernels:
 * the reference's camera::ray_color loop (core/src/cameras/camera.cuh:149-264) with a PCG32 stream per
 * (pixel, sample), spp samples per pixel, non-finite samples dropped, and otherwise the reference's
 * rules:
 *   - perspective_camera::get_ray with the thin lens and a time sample (perspective_camera.cuh:112-117);
 *   - sphere (strict interval), quad and directional light (inclusive), triangle (Moller-Trumbore,
 *     |det| < 1e-6 rejected) intersections, tmin 1e-5 (sphere.cuh:111-166, quad.cuh:100-133,
 *     directional_light.cuh:76-120, triangle.cuh:130-185, camera.cuh:161);
 *   - invisible lights hidden from primary rays; a one-sided light seen from behind re-hits from
 *     t + 0.001 (directional_light.cuh:106, camera.cuh:177-190);
 *   - lambertian: 50/50 mixture of light-list sampling (light 0 sampled, pdf averaged over all lights,
 *     hittable_list.cuh:173-215) and cosine sampling, or cosine sampling alone with no lights;
 *     metal: reflect + fuzz * unit-sphere sample; dielectric with Schlick (lambertian.cuh:63-143,
 *     metal.cuh:52-64, dielectric.cuh:32-63);
 *   - solid / checker / image textures, constant / sky-gradient / equirectangular backgrounds.
 * All geometry and shading arithmetic is in double.  The random draws are the clean kernels' PCG32
 * draws (24-bit uniforms), so a sample starts on the same path as the kernel's and drifts away only
 * where rounding differs.  Closest hits are found by testing every primitive, or, in scenes of more
 * than BVH_MIN_PRIMS primitives, through a median-split bounding-volume tree of double-precision boxes
 * (padded outward, so it finds the same closest hit; only exact-distance ties may resolve differently).
 *
 * Exported C API (ctypes, tests/oracles.py): f64_scene_create / f64_scene_destroy / f64_render.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rtc.h"

#define PI 3.14159265358979323846

typedef struct { double x, y, z; } d3;
static inline d3 D(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 Dp(const float* p) { return D(p[0], p[1], p[2]); }
static inline d3 add(d3 a, d3 b) { return D(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 sub(d3 a, d3 b) { return D(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 mul(double s, d3 a) { return D(s * a.x, s * a.y, s * a.z); }
static inline d3 neg(d3 a) { return D(-a.x, -a.y, -a.z); }
static inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 cross(d3 a, d3 b) { return D(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double len(d3 a) { return sqrt(dot(a, a)); }
static inline d3 unit(d3 a) { return mul(1.0 / len(a), a); }
static inline d3 at(d3 o, d3 d, double t) { return add(o, mul(t, d)); }
static inline d3 reflect(d3 i, d3 n) { return sub(i, mul(2.0 * dot(n, i), n)); }
static inline d3 refract(d3 i, d3 n, double eta) {
    double dv = dot(n, i);
    double k = 1.0 - eta * eta * (1.0 - dv * dv);
    if (k < 0.0) return D(0, 0, 0);
    return sub(mul(eta, i), mul(eta * dv + sqrt(k), n));
}

/* ---- PCG32, the clean kernels' stream ------------------------------------------------------------ */
typedef struct { uint64_t state, inc; } pcg_t;
static inline uint32_t pcg_next(pcg_t* r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ull + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
static inline void pcg_seed(pcg_t* r, uint64_t init, uint64_t seq) {
    r->state = 0u;
    r->inc = (seq << 1u) | 1u;
    pcg_next(r);
    r->state += init;
    pcg_next(r);
}
static inline double U(pcg_t* r) { return (double)(pcg_next(r) >> 8) * (1.0 / 16777216.0); }
static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* ---- scene ---------------------------------------------------------------------------------------- */
enum { K_LIGHT = 0, K_SPHERE = 1, K_QUAD = 2, K_TRI = 3 };
typedef struct {
    int kind, mat;
    d3 a, b, c;          /* sphere: centre, (r, -, -); planar: Q/P, u, v; triangle: v0, e1, e2 */
    double r;
    d3 n, w;             /* planar: unit normal, w; triangle: flat normal */
    double D, area;
    int invisible;       /* lights */
    int smooth;
    d3 vn[3];
    double uv[6];        /* triangle: per-vertex texture coordinates (zeros without) */
} prim_t;
typedef struct { int kind; double col[3]; double inv_scale; int even, odd, image; } tex_t;
typedef struct { int kind; int tex; double fuzz, ior, intensity; int directional; } mat_t;
typedef struct { const uint8_t* px; int w, h; } img_t;
typedef struct {
    prim_t* prims;
    int np, nlights;     /* lights are prims[0 .. nlights) */
    tex_t* tex;
    int ntex;
    mat_t* mat;
    int nmat;
    img_t* img;
    int nimg;
    uint8_t* img_bytes;
    d3 cam_origin, llc, horizontal, vertical, cu, cv;
    double lens;
    int bg_kind;
    double bg[3], top[3];
    float* env;
    int env_w, env_h;
    struct bvh_node* nodes;   /* NULL: brute force */
    int* order;               /* leaf order of primitive indices */
} scene_t;

/* ---- bounding-volume tree (large scenes) ---------------------------------------------------------- */
#define BVH_MIN_PRIMS 64
#define BVH_LEAF 4
typedef struct bvh_node {
    double lo[3], hi[3];
    int left, count;   /* count > 0: leaf of order[left .. left+count); else children left, left+1 */
} bvh_node;

static void bvh_create(scene_t* s);

static void planar(prim_t* p, d3 q, d3 u, d3 v) {
    p->a = q;
    p->b = u;
    p->c = v;
    d3 n = cross(u, v);
    p->n = unit(n);
    p->D = dot(p->n, q);
    p->w = mul(1.0 / dot(n, n), n);
    p->area = len(n);
}

void* f64_scene_create(const rtc_scene_desc* d) {
    scene_t* s = (scene_t*)calloc(1, sizeof(scene_t));
    uint64_t ntri = 0;
    for (uint32_t i = 0; i < d->num_meshes; ++i) ntri += d->meshes[i].num_triangles;
    s->np = (int)(d->num_dir_lights + d->num_spheres + d->num_quads + ntri);
    s->nlights = (int)d->num_dir_lights;
    s->prims = (prim_t*)calloc((size_t)s->np + 1, sizeof(prim_t));
    s->ntex = (int)(d->num_textures + d->num_dir_lights);
    s->tex = (tex_t*)calloc((size_t)s->ntex + 1, sizeof(tex_t));
    s->nmat = (int)(d->num_materials + d->num_dir_lights);
    s->mat = (mat_t*)calloc((size_t)s->nmat + 1, sizeof(mat_t));
    for (uint32_t i = 0; i < d->num_textures; ++i) {
        const rtc_texture* t = &d->textures[i];
        tex_t* o = &s->tex[i];
        o->kind = t->kind;
        for (int k = 0; k < 3; ++k) o->col[k] = t->color[k];
        o->inv_scale = t->kind == RTC_TEX_CHECKER ? 1.0 / (double)t->scale : 0.0;
        o->even = t->even;
        o->odd = t->odd;
        o->image = t->image;
    }
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        const rtc_material* m = &d->materials[i];
        mat_t* o = &s->mat[i];
        o->kind = m->kind;
        o->tex = m->texture;
        o->fuzz = m->fuzz < 1.0f ? m->fuzz : 1.0;
        o->ior = m->ior;
        o->intensity = m->intensity;
        o->directional = m->directional;
    }
    s->nimg = (int)d->num_images;
    s->img = (img_t*)calloc((size_t)s->nimg + 1, sizeof(img_t));
    for (uint32_t i = 0; i < d->num_images; ++i) {
        size_t nb = (size_t)d->images[i].width * d->images[i].height * 3;
        uint8_t* px = (uint8_t*)malloc(nb);
        memcpy(px, d->images[i].rgb, nb);
        s->img[i].px = px;
        s->img[i].w = d->images[i].width;
        s->img[i].h = d->images[i].height;
    }
    int k = 0;
    for (uint32_t i = 0; i < d->num_dir_lights; ++i, ++k) {
        const rtc_dir_light* L = &d->dir_lights[i];
        prim_t* p = &s->prims[k];
        p->kind = K_LIGHT;
        planar(p, Dp(L->position), Dp(L->u), Dp(L->v));
        p->invisible = L->invisible;
        int ti = (int)d->num_textures + (int)i, mi = (int)d->num_materials + (int)i;
        s->tex[ti].kind = RTC_TEX_SOLID;
        for (int c = 0; c < 3; ++c) s->tex[ti].col[c] = L->color[c];
        s->mat[mi].kind = RTC_MAT_DIFFUSE_LIGHT;
        s->mat[mi].tex = ti;
        s->mat[mi].intensity = L->intensity;
        s->mat[mi].directional = 1;
        p->mat = mi;
    }
    for (uint32_t i = 0; i < d->num_spheres; ++i, ++k) {
        prim_t* p = &s->prims[k];
        p->kind = K_SPHERE;
        p->a = Dp(d->spheres[i].center);
        p->r = d->spheres[i].radius;
        p->mat = d->spheres[i].material;
    }
    for (uint32_t i = 0; i < d->num_quads; ++i, ++k) {
        prim_t* p = &s->prims[k];
        p->kind = K_QUAD;
        planar(p, Dp(d->quads[i].q), Dp(d->quads[i].u), Dp(d->quads[i].v));
        p->mat = d->quads[i].material;
    }
    for (uint32_t m = 0; m < d->num_meshes; ++m) {
        const rtc_mesh* M = &d->meshes[m];
        for (uint32_t f = 0; f < M->num_triangles; ++f, ++k) {
            prim_t* p = &s->prims[k];
            uint32_t ia = M->indices[3 * f], ib = M->indices[3 * f + 1], ic = M->indices[3 * f + 2];
            d3 a = Dp(M->vertices + 3 * ia), b = Dp(M->vertices + 3 * ib), c = Dp(M->vertices + 3 * ic);
            p->kind = K_TRI;
            p->a = a;
            p->b = sub(b, a);
            p->c = sub(c, a);
            p->n = unit(cross(sub(a, b), sub(a, c)));   /* triangle.cuh:87-123 middle normal */
            p->mat = M->material;
            p->smooth = M->smooth && M->normals;
            if (p->smooth) {
                p->vn[0] = unit(Dp(M->normals + 3 * ia));
                p->vn[1] = unit(Dp(M->normals + 3 * ib));
                p->vn[2] = unit(Dp(M->normals + 3 * ic));
            }
            if (M->uvs) {
                const uint32_t vi[3] = {ia, ib, ic};
                for (int q = 0; q < 3; ++q) {
                    p->uv[2 * q] = M->uvs[2 * vi[q]];
                    p->uv[2 * q + 1] = M->uvs[2 * vi[q] + 1];
                }
            }
        }
    }
    /* camera: perspective_camera::initialize (perspective_camera.cuh:41-108) */
    const rtc_camera* C = &d->camera;
    double theta = C->vfov * PI / 180.0, hh = tan(theta / 2.0), hw = C->aspect * hh, focus = C->focus;
    d3 lf = Dp(C->look_from), la = Dp(C->look_at), up = Dp(C->up);
    d3 w = unit(sub(lf, la)), u = unit(cross(up, w)), v = cross(w, u);
    s->cam_origin = lf;
    s->llc = sub(sub(sub(lf, mul(hw * focus, u)), mul(hh * focus, v)), mul(focus, w));
    s->horizontal = mul(2.0 * hw * focus, u);
    s->vertical = mul(2.0 * hh * focus, v);
    s->cu = u;
    s->cv = v;
    s->lens = C->aperture / 2.0;
    s->bg_kind = d->background.kind;
    for (int c = 0; c < 3; ++c) {
        s->bg[c] = d->background.color[c];
        s->top[c] = d->background.top[c];
    }
    if (d->background.kind == RTC_BG_ENV_MAP) {
        size_t n = (size_t)d->background.env_width * d->background.env_height * 3;
        s->env = (float*)malloc(n * sizeof(float));
        memcpy(s->env, d->background.env_rgb, n * sizeof(float));
        s->env_w = d->background.env_width;
        s->env_h = d->background.env_height;
    }
    bvh_create(s);
    return s;
}

static void prim_box(const prim_t* p, double lo[3], double hi[3]) {
    d3 pts[4];
    int n = 0;
    if (p->kind == K_SPHERE) {
        const double c[3] = {p->a.x, p->a.y, p->a.z};
        for (int k = 0; k < 3; ++k) { lo[k] = c[k] - fabs(p->r); hi[k] = c[k] + fabs(p->r); }
        return;
    }
    if (p->kind == K_TRI) {
        pts[0] = p->a; pts[1] = add(p->a, p->b); pts[2] = add(p->a, p->c); n = 3;
    } else if (p->kind == K_QUAD) {
        pts[0] = p->a; pts[1] = add(p->a, p->b); pts[2] = add(p->a, p->c); pts[3] = add(pts[1], p->c); n = 4;
    } else {   /* light: centred quad */
        d3 h = add(mul(0.5, p->b), mul(0.5, p->c)), g = sub(mul(0.5, p->b), mul(0.5, p->c));
        pts[0] = sub(p->a, h); pts[1] = add(p->a, h); pts[2] = sub(p->a, g); pts[3] = add(p->a, g); n = 4;
    }
    for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
    for (int i = 0; i < n; ++i) {
        const double v[3] = {pts[i].x, pts[i].y, pts[i].z};
        for (int k = 0; k < 3; ++k) { if (v[k] < lo[k]) lo[k] = v[k]; if (v[k] > hi[k]) hi[k] = v[k]; }
    }
}

typedef struct { double key; int idx; } keyed_t;
static int cmp_keyed(const void* a, const void* b) {
    const keyed_t *x = (const keyed_t*)a, *y = (const keyed_t*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx ? 1 : 0);
}

static int bvh_build(scene_t* s, double* lo, double* hi, double* cen, keyed_t* tmp, int first, int count, int* nn) {
    const int me = (*nn)++;
    bvh_node* nd = &s->nodes[me];
    for (int k = 0; k < 3; ++k) { nd->lo[k] = INFINITY; nd->hi[k] = -INFINITY; }
    double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = first; i < first + count; ++i) {
        const int q = s->order[i];
        for (int k = 0; k < 3; ++k) {
            if (lo[3 * q + k] < nd->lo[k]) nd->lo[k] = lo[3 * q + k];
            if (hi[3 * q + k] > nd->hi[k]) nd->hi[k] = hi[3 * q + k];
            if (cen[3 * q + k] < clo[k]) clo[k] = cen[3 * q + k];
            if (cen[3 * q + k] > chi[k]) chi[k] = cen[3 * q + k];
        }
    }
    for (int k = 0; k < 3; ++k) {   /* outward padding: flat boxes and rounding of the slab test */
        const double pad = 1e-9 * (fabs(nd->lo[k]) + fabs(nd->hi[k]) + 1.0);
        nd->lo[k] -= pad;
        nd->hi[k] += pad;
    }
    if (count <= BVH_LEAF) {
        nd->left = first;
        nd->count = count;
        return me;
    }
    int axis = 0;
    for (int k = 1; k < 3; ++k)
        if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
    /* sort the span by centroid on the widest axis (scene creation may run on several threads at once,
       so no global sort state) */
    for (int i = 0; i < count; ++i) {
        tmp[i].idx = s->order[first + i];
        tmp[i].key = cen[3 * tmp[i].idx + axis];
    }
    qsort(tmp, (size_t)count, sizeof(keyed_t), cmp_keyed);
    for (int i = 0; i < count; ++i) s->order[first + i] = tmp[i].idx;
    const int half = count / 2;
    nd->count = 0;
    const int l = bvh_build(s, lo, hi, cen, tmp, first, half, nn);
    const int r = bvh_build(s, lo, hi, cen, tmp, first + half, count - half, nn);
    (void)l;
    s->nodes[me].left = l;
    s->nodes[me].count = -r;   /* children l and r */
    return me;
}

static int g_bvh_min = BVH_MIN_PRIMS;
/* Scenes created afterwards use the tree above `min_prims` primitives (a huge value: brute force always). */
void f64_set_bvh_threshold(int min_prims) { g_bvh_min = min_prims; }

static void bvh_create(scene_t* s) {
    if (s->np <= g_bvh_min) return;
    double* lo = (double*)malloc(sizeof(double) * 3 * (size_t)s->np);
    double* hi = (double*)malloc(sizeof(double) * 3 * (size_t)s->np);
    double* cen = (double*)malloc(sizeof(double) * 3 * (size_t)s->np);
    s->order = (int*)malloc(sizeof(int) * (size_t)s->np);
    s->nodes = (bvh_node*)calloc(2 * (size_t)s->np, sizeof(bvh_node));
    for (int i = 0; i < s->np; ++i) {
        prim_box(&s->prims[i], lo + 3 * i, hi + 3 * i);
        for (int k = 0; k < 3; ++k) cen[3 * i + k] = 0.5 * (lo[3 * i + k] + hi[3 * i + k]);
        s->order[i] = i;
    }
    keyed_t* tmp = (keyed_t*)malloc(sizeof(keyed_t) * (size_t)s->np);
    int nn = 0;
    bvh_build(s, lo, hi, cen, tmp, 0, s->np, &nn);
    free(tmp);
    free(lo);
    free(hi);
    free(cen);
}

void f64_scene_destroy(void* p) {
    scene_t* s = (scene_t*)p;
    if (!s) return;
    free(s->nodes);
    free(s->order);
    for (int i = 0; i < s->nimg; ++i) free((void*)s->img[i].px);
    free(s->img);
    free(s->prims);
    free(s->tex);
    free(s->mat);
    free(s->env);
    free(s);
}

/* ---- intersection --------------------------------------------------------------------------------- */
static int planar_t(const prim_t* p, d3 o, d3 d, double tmin, double tmax, int centred, double* t, double* al,
                    double* be) {
    double denom = dot(p->n, d);
    if (fabs(denom) < 1e-8) return 0;
    double tt = (p->D - dot(p->n, o)) / denom;
    if (!(tmin <= tt && tt <= tmax)) return 0;
    d3 pl = sub(at(o, d, tt), p->a);
    double a = dot(p->w, cross(pl, p->c)), b = dot(p->w, cross(p->b, pl));
    if (centred) {
        if (a < -0.5 || a > 0.5 || b < -0.5 || b > 0.5) return 0;
    } else if (a < 0.0 || a > 1.0 || b < 0.0 || b > 1.0) {
        return 0;
    }
    *t = tt;
    *al = a;
    *be = b;
    return 1;
}

static int prim_t_test(const prim_t* p, d3 o, d3 d, double tmin, double tmax, int hide, double* t) {
    double a, b;
    switch (p->kind) {
    case K_SPHERE: {
        d3 oc = sub(o, p->a);
        double aa = dot(d, d), hb = dot(oc, d), cc = dot(oc, oc) - p->r * p->r;
        double disc = hb * hb - aa * cc;
        if (disc < 0.0) return 0;
        double sq = sqrt(disc), root = (-hb - sq) / aa;
        if (!(tmin < root && root < tmax)) {
            root = (-hb + sq) / aa;
            if (!(tmin < root && root < tmax)) return 0;
        }
        *t = root;
        return 1;
    }
    case K_QUAD:
        return planar_t(p, o, d, tmin, tmax, 0, t, &a, &b);
    case K_LIGHT:
        if (!planar_t(p, o, d, tmin, tmax, 1, t, &a, &b)) return 0;
        return !(p->invisible && hide);
    default: {
        d3 pv = cross(d, p->c);
        double det = dot(p->b, pv);
        if (fabs(det) < 1e-6) return 0;
        double inv = 1.0 / det;
        d3 tv = sub(o, p->a);
        double u = dot(tv, pv) * inv;
        if (u < 0.0 || u > 1.0) return 0;
        d3 qv = cross(tv, p->b);
        double v = dot(d, qv) * inv;
        if (v < 0.0 || u + v > 1.0) return 0;
        double tt = dot(p->c, qv) * inv;
        if (tt < tmin || tt > tmax) return 0;
        *t = tt;
        return 1;
    }
    }
}

static int slab(const bvh_node* nd, const double o[3], const double inv[3], double tmin, double tmax) {
    for (int k = 0; k < 3; ++k) {
        double t0 = (nd->lo[k] - o[k]) * inv[k], t1 = (nd->hi[k] - o[k]) * inv[k];
        if (t0 > t1) { double x = t0; t0 = t1; t1 = x; }
        if (t0 != t0) t0 = -INFINITY;   /* 0 * inf: the ray lies in the slab's plane */
        if (t1 != t1) t1 = INFINITY;
        if (t0 > tmin) tmin = t0;
        if (t1 < tmax) tmax = t1;
        if (tmax < tmin) return 0;
    }
    return 1;
}

static int closest(const scene_t* s, d3 o, d3 d, double tmin, double tmax, int hide, double* tout) {
    int best = -1;
    double bt = tmax, t;
    if (!s->nodes) {
        for (int i = 0; i < s->np; ++i)
            if (prim_t_test(&s->prims[i], o, d, tmin, bt, hide, &t)) {
                bt = t;
                best = i;
            }
        *tout = bt;
        return best;
    }
    const double oo[3] = {o.x, o.y, o.z};
    const double inv[3] = {1.0 / d.x, 1.0 / d.y, 1.0 / d.z};
    int stack[128], sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const bvh_node* nd = &s->nodes[stack[--sp]];
        if (!slab(nd, oo, inv, tmin, bt)) continue;
        if (nd->count > 0) {
            for (int i = nd->left; i < nd->left + nd->count; ++i) {
                const int q = s->order[i];
                if (prim_t_test(&s->prims[q], o, d, tmin, bt, hide, &t)) {
                    bt = t;
                    best = q;
                }
            }
        } else if (sp + 2 <= 128) {
            stack[sp++] = -nd->count;
            stack[sp++] = nd->left;
        }
    }
    *tout = bt;
    return best;
}

typedef struct { d3 p, n; double u, v; int front, mat; } hit_t;

static void finalize(const scene_t* s, int pi, double t, d3 o, d3 d, hit_t* h) {
    const prim_t* p = &s->prims[pi];
    h->p = at(o, d, t);
    h->mat = p->mat;
    d3 outward;
    if (p->kind == K_SPHERE) {
        outward = mul(1.0 / p->r, sub(h->p, p->a));
        double theta = acos(-outward.y), phi = atan2(-outward.z, outward.x) + PI;
        h->u = fmod(phi / (2.0 * PI), 1.0);
        h->v = fmod(theta / PI, 1.0);
    } else if (p->kind == K_QUAD || p->kind == K_LIGHT) {
        d3 pl = sub(h->p, p->a);
        double a = dot(p->w, cross(pl, p->c)), b = dot(p->w, cross(p->b, pl));
        outward = p->n;
        h->u = p->kind == K_QUAD ? a : a + 0.5;
        h->v = p->kind == K_QUAD ? b : b + 0.5;
    } else {
        outward = p->n;
        if (p->smooth) {
            d3 pv = cross(d, p->c);
            double inv = 1.0 / dot(p->b, pv);
            d3 tv = sub(o, p->a);
            double bu = dot(tv, pv) * inv, bv = dot(d, cross(tv, p->b)) * inv, bc = 1.0 - bu - bv;
            outward = add(add(mul(bu, p->vn[1]), mul(bv, p->vn[2])), mul(bc, p->vn[0]));
        }
        /* get_triangle_uv at the hit point (barycentric interpolation of the vertex uvs, wrapped into
           [0, 1): math_utils.cuh:73-86, uvmapping.cuh:415-447) */
        d3 p2 = sub(h->p, p->a);
        double d00 = dot(p->b, p->b), d01 = dot(p->b, p->c), d11 = dot(p->c, p->c);
        double d20 = dot(p2, p->b), d21 = dot(p2, p->c), den = d00 * d11 - d01 * d01;
        double bv = (d11 * d20 - d01 * d21) / den, bw = (d00 * d21 - d01 * d20) / den, bu = 1.0 - bv - bw;
        double tu = fmod(bu * p->uv[0] + bv * p->uv[2] + bw * p->uv[4], 1.0);
        double tv = fmod(bu * p->uv[1] + bv * p->uv[3] + bw * p->uv[5], 1.0);
        h->u = tu < 0.0 ? tu + 1.0 : tu;
        h->v = tv < 0.0 ? tv + 1.0 : tv;
    }
    h->front = dot(d, outward) < 0.0;
    h->n = h->front ? outward : neg(outward);
}

/* ---- textures, background, light pdf -------------------------------------------------------------- */
static void tex_value(const scene_t* s, int ti, double u, double v, d3 p, double* c) {
    for (int guard = 0; guard < 8 && ti >= 0 && ti < s->ntex; ++guard) {
        const tex_t* t = &s->tex[ti];
        if (t->kind == RTC_TEX_SOLID) {
            c[0] = t->col[0], c[1] = t->col[1], c[2] = t->col[2];
            return;
        }
        if (t->kind == RTC_TEX_CHECKER) {
            long xi = (long)floor(t->inv_scale * p.x), yi = (long)floor(t->inv_scale * p.y),
                 zi = (long)floor(t->inv_scale * p.z);
            ti = ((xi + yi + zi) % 2 == 0) ? t->even : t->odd;
            continue;
        }
        const img_t* im = &s->img[t->image];
        double uu = u < 0 ? 0 : (u > 1 ? 1 : u), vv = 1.0 - (v < 0 ? 0 : (v > 1 ? 1 : v));
        int i = (int)(uu * im->w), j = (int)(vv * im->h);
        i = i < 0 ? 0 : (i < im->w ? i : im->w - 1);
        j = j < 0 ? 0 : (j < im->h ? j : im->h - 1);
        const uint8_t* px = im->px + ((size_t)j * im->w + i) * 3;
        for (int k = 0; k < 3; ++k) c[k] = px[k] / 255.0;
        return;
    }
    c[0] = c[1] = c[2] = 0.0;
}

static void background(const scene_t* s, d3 dir, double* c) {
    if (s->bg_kind == RTC_BG_CONSTANT) {
        for (int k = 0; k < 3; ++k) c[k] = s->bg[k];
        return;
    }
    d3 u = unit(dir);
    if (s->bg_kind == RTC_BG_SKY_GRADIENT) {
        double a = 0.5 * (u.y + 1.0);
        for (int k = 0; k < 3; ++k) c[k] = (1.0 - a) * s->bg[k] + a * s->top[k];
        return;
    }
    double theta = acos(-u.y), phi = atan2(-u.z, u.x) + PI;
    int x = (int)(phi / (2.0 * PI) * s->env_w), y = (int)((1.0 - theta / PI) * s->env_h);
    x = x < 0 ? 0 : (x >= s->env_w ? s->env_w - 1 : x);
    y = y < 0 ? 0 : (y >= s->env_h ? s->env_h - 1 : y);
    const float* px = s->env + 3 * ((size_t)y * s->env_w + x);
    for (int k = 0; k < 3; ++k) c[k] = px[k];
}

static double lights_pdf(const scene_t* s, d3 o, d3 v) {
    double sum = 0.0, wgt = 1.0 / s->nlights;
    for (int i = 0; i < s->nlights; ++i) {
        const prim_t* L = &s->prims[i];
        double t, a, b;
        if (!planar_t(L, o, v, 1e-5, INFINITY, 1, &t, &a, &b)) continue;
        d3 nrm = dot(v, L->n) < 0.0 ? L->n : neg(L->n);
        double cosine = fabs(dot(v, nrm) / len(v));
        sum += wgt * (t * t * dot(v, v)) / (cosine * L->area);
    }
    return sum;
}

/* ---- one sample ----------------------------------------------------------------------------------- */
static void sample(const scene_t* s, d3 o, d3 d, int max_depth, pcg_t* rng, double* out) {
    double res[3] = {0, 0, 0}, att[3] = {1, 1, 1};
    for (int depth = max_depth; depth > 0; --depth) {
        const int hide = depth == max_depth;
        double t;
        int pi = closest(s, o, d, 1e-5, 3.402823466e+38, hide, &t);
        if (pi < 0) {
            double bg[3];
            background(s, d, bg);
            for (int k = 0; k < 3; ++k) res[k] += att[k] * bg[k];
            break;
        }
        hit_t h;
        finalize(s, pi, t, o, d, &h);
        const mat_t* m = &s->mat[h.mat];
        double em[3] = {0, 0, 0};
        if (m->kind == RTC_MAT_DIFFUSE_LIGHT) {
            if (m->directional && !h.front) {
                double t2;   /* one-sided light seen from behind: re-hit past it, emission stays 0 */
                int p2 = closest(s, o, d, t + 0.001, 3.402823466e+38, hide, &t2);
                if (p2 >= 0) {
                    finalize(s, p2, t2, o, d, &h);
                    m = &s->mat[h.mat];
                }
            } else {
                double tv[3];
                tex_value(s, m->tex, h.u, h.v, h.p, tv);
                for (int k = 0; k < 3; ++k) em[k] = tv[k] * m->intensity;
            }
        }
        for (int k = 0; k < 3; ++k) res[k] += att[k] * em[k];
        if (m->kind == RTC_MAT_DIFFUSE_LIGHT) break;
        if (m->kind == RTC_MAT_METAL) {
            double a[3];
            tex_value(s, m->tex, h.u, h.v, h.p, a);
            d3 rs;
            do {
                double x = U(rng), y = U(rng), z = U(rng);
                rs = D(2 * x - 1, 2 * y - 1, 2 * z - 1);
            } while (dot(rs, rs) >= 1.0);
            d = add(reflect(unit(d), h.n), mul(m->fuzz, rs));
            o = h.p;
            for (int k = 0; k < 3; ++k) att[k] *= a[k];
            continue;
        }
        if (m->kind == RTC_MAT_DIELECTRIC) {
            double ratio = h.front ? 1.0 / m->ior : m->ior;
            d3 ud = unit(d);
            double ct = dot(neg(ud), h.n), cs = ct < 1.0 ? ct : 1.0, sn = sqrt(1.0 - cs * cs);
            int refl = ratio * sn > 1.0;
            if (!refl) {
                double r0 = (1.0 - ratio) / (1.0 + ratio);
                r0 *= r0;
                refl = r0 + (1.0 - r0) * pow(1.0 - cs, 5.0) > U(rng);
            }
            d = refl ? reflect(ud, h.n) : refract(ud, h.n, ratio);
            o = h.p;
            continue;
        }
        /* lambertian */
        double a[3];
        tex_value(s, m->tex, h.u, h.v, h.p, a);
        d3 w = unit(h.n);
        d3 ax = fabs(w.x) > 0.9 ? D(0, 1, 0) : D(1, 0, 0);
        d3 bv = unit(cross(w, ax)), bu = cross(w, bv);
        d3 dir;
        double pdf;
        if (s->nlights > 0) {
            if (U(rng) < 0.5) {
                if (s->nlights > 1) (void)U(rng);   /* get_int: one draw, light 0 */
                const prim_t* L = &s->prims[0];
                double ru = U(rng), rv = U(rng);
                dir = sub(add(add(L->a, mul(ru - 0.5, L->b)), mul(rv - 0.5, L->c)), h.p);
            } else {
                double r1 = U(rng), r2 = U(rng), phi = 2.0 * PI * r1, z = sqrt(1.0 - r2), r2s = sqrt(r2);
                dir = add(add(mul(cos(phi) * r2s, bu), mul(sin(phi) * r2s, bv)), mul(z, w));
            }
            double cv = dot(unit(dir), w) / PI;
            pdf = 0.5 * lights_pdf(s, h.p, dir) + 0.5 * (cv > 0.0 ? cv : 0.0);
        } else {
            double r1 = U(rng), r2 = U(rng), phi = 2.0 * PI * r1, z = sqrt(1.0 - r2), r2s = sqrt(r2);
            dir = add(add(mul(cos(phi) * r2s, bu), mul(sin(phi) * r2s, bv)), mul(z, w));
            double cv = dot(unit(dir), w) / PI;
            pdf = cv > 0.0 ? cv : 0.0;
        }
        double cst = dot(h.n, unit(dir));
        double spdf = cst < 0.0 ? 0.0 : cst / PI;
        for (int k = 0; k < 3; ++k) att[k] *= a[k] * spdf / pdf;
        o = h.p;
        d = dir;
    }
    for (int k = 0; k < 3; ++k) out[k] = res[k];
}

/* ---- pixels --------------------------------------------------------------------------------------- */
typedef struct {
    const scene_t* s;
    int width, height, spp, max_depth;
    uint32_t seed;
    const int64_t* pixels;
    int64_t n, begin, end;
    double* out;
} job_t;

static void* worker(void* arg) {
    job_t* J = (job_t*)arg;
    const scene_t* s = J->s;
    for (int64_t k = J->begin; k < J->end; ++k) {
        const int64_t pix = J->pixels[k];
        const int i = (int)(pix % J->width), j = (int)(pix / J->width);
        double acc[3] = {0, 0, 0};
        for (int smp = 0; smp < J->spp; ++smp) {
            pcg_t r;
            pcg_seed(&r, mix64(((uint64_t)J->seed << 32) ^ (uint64_t)pix), (uint64_t)smp);
            double u = (i + U(&r)) / J->width, v = (j + U(&r)) / J->height;
            double dx, dy;
            do {
                dx = 2 * U(&r) - 1;
                dy = 2 * U(&r) - 1;
            } while (dx * dx + dy * dy >= 1.0);
            d3 off = add(mul(s->lens * dx, s->cu), mul(s->lens * dy, s->cv));
            (void)U(&r);   /* the time sample */
            d3 o = add(s->cam_origin, off);
            d3 d = sub(sub(add(add(s->llc, mul(u, s->horizontal)), mul(v, s->vertical)), s->cam_origin), off);
            double c[3];
            sample(s, o, d, J->max_depth, &r, c);
            if (isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2]))
                for (int k2 = 0; k2 < 3; ++k2) acc[k2] += c[k2];
        }
        for (int k2 = 0; k2 < 3; ++k2) J->out[3 * k + k2] = acc[k2];
    }
    return NULL;
}

/* Renders `n` pixels (frame-buffer indices j*width + i) with `spp` clean-mode samples each; writes the
 * radiance sums (n x 3 doubles) to out.  Returns 0. */
int f64_render(void* scene, int width, int height, int spp, int max_depth, uint32_t seed, const int64_t* pixels,
               int64_t n, double* out, int threads) {
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    job_t jobs[256];
    for (int t = 0; t < threads; ++t) {
        jobs[t] = (job_t){(const scene_t*)scene, width, height, spp, max_depth, seed, pixels, n, n * t / threads,
                          n * (t + 1) / threads, out};
        pthread_create(&th[t], NULL, worker, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    return 0;
}
