/*
 * rt_port.c - TEST INFRASTRUCTURE ONLY (the oracle).  Never part of the product path.
 *
 * A plain-C restatement of the reference's per-sample path-tracing path (flarive/CortexRaytracerCuda,
 * core/src/...), driven by the same rtc_scene_desc as the product.  Each function cites the reference
 * code it restates.  Float expressions keep the reference's operation order; build with
 * -ffp-contract=off (oracle/Makefile) so roundings match a plain g++ build of the reference.
 * Transcendentals call glibc's float functions, as the reference's host build does.
 *
 * Pinned against the reference itself: tests/golden/ holds outputs of the reference's own classes
 * (oracle/_ref/libref_cpu.so, generated by tests/golden/make_golden.py) and tests/test_oracle_port.py
 * checks this port against them.
 *
 * Differences from the reference that do not change results: the BVH is a median-split tree of this
 * file's own (the reference's is random-axis with an exchange sort, bvh_node.cuh:63-108); only the
 * order of exactly-equal-t candidates can differ.
 *
 * Exported: port_scene_create / port_scene_destroy / port_render_pixels / port_trace_closest /
 * port_rng_draws / port_set_trig / port_last_error.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <stdio.h>

#include "rtc.h"

#define PI_F 3.14159265358979323846f   /* the reference's float M_PI (misc/constants.cuh:35) */

static __thread char g_err[256];

/* Transcendental evaluation: 0 = glibc's float functions (cosf, sinf, acosf, atan2f), as a g++ build
 * of the reference calls them; 1 = evaluated in double and rounded to float, as the product's
 * compat kernels do on the device.  The two differ only in the last ulp of these four functions. */
static int g_trig = 0;
void port_set_trig(int mode) { g_trig = mode; }
static inline float f_cos(float x) { return g_trig ? (float)cos((double)x) : cosf(x); }
static inline float f_sin(float x) { return g_trig ? (float)sin((double)x) : sinf(x); }
static inline float f_acos(float x) { return g_trig ? (float)acos((double)x) : acosf(x); }
static inline float f_atan2(float y, float x) { return g_trig ? (float)atan2((double)y, (double)x) : atan2f(y, x); }
static inline float f_pow(float x, float y) { return g_trig ? (float)pow((double)x, (double)y) : powf(x, y); }

/* ---------------------------------------------------------------------------------------------- */
/* vectors: glm semantics (func_geometric.inl), misc/vector3.cuh                                  */
/* ---------------------------------------------------------------------------------------------- */
typedef struct { float x, y, z; } v3;
static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 Vp(const float* p) { return V(p[0], p[1], p[2]); }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline v3 vscale(float s, v3 a) { return V(s * a.x, s * a.y, s * a.z); }
static inline v3 vdivs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static inline float vdot(v3 a, v3 b) { float tx = a.x * b.x, ty = a.y * b.y, tz = a.z * b.z; return tx + ty + tz; }
static inline v3 vcross(v3 x, v3 y) {
    return V(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
static inline float vlensq(v3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }   /* vector_length_squared */
static inline float vlen(v3 v) { return sqrtf(vlensq(v)); }
static inline v3 vunit(v3 v) { float l = sqrtf(vlensq(v)); return V(v.x / l, v.y / l, v.z / l); }   /* unit_vector */
static inline v3 vreflect(v3 I, v3 N) { float d = vdot(N, I); v3 nd = V(N.x * d, N.y * d, N.z * d); return vsub(I, V(nd.x * 2.0f, nd.y * 2.0f, nd.z * 2.0f)); }
static inline v3 vrefract(v3 I, v3 N, float eta) {
    float dv = vdot(N, I);
    float k = 1.0f - eta * eta * (1.0f - dv * dv);
    if (k >= 0.0f) { float s = eta * dv + sqrtf(k); return vsub(vscale(eta, I), vscale(s, N)); }
    return V(0.0f, 0.0f, 0.0f);
}
static inline v3 vat(v3 o, v3 d, float t) { return vadd(o, vscale(t, d)); }   /* ray::at */

/* ---------------------------------------------------------------------------------------------- */
/* random numbers: thrust minstd_rand + uniform_real_distribution<float>(0,1)                      */
/* ---------------------------------------------------------------------------------------------- */
typedef struct { int clean; uint32_t x; uint64_t st, inc; } rng_t;
static inline void minstd_seed(rng_t* r, uint32_t s) { uint32_t m = s % 2147483647u; r->clean = 0; r->x = m ? m : 1u; }
static inline float minstd_uniform(rng_t* r) {
    r->x = (uint32_t)(((uint64_t)r->x * 48271ull) % 2147483647ull);
    return (float)(r->x - 1u) / (1.0f + (float)(2147483646u - 1u));
}
/* PCG32 XSH-RR (O'Neill 2014) for clean mode, seeded like the product's clean kernel */
static inline uint32_t pcg_next(rng_t* r) {
    uint64_t old = r->st;
    r->st = old * 6364136223846793005ull + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u), rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
static inline void pcg_seed(rng_t* r, uint64_t init, uint64_t seq) {
    r->clean = 1; r->st = 0; r->inc = (seq << 1u) | 1u; pcg_next(r); r->st += init; pcg_next(r);
}
static inline float U(rng_t* r) {
    if (r->clean) return (float)(pcg_next(r) >> 8) * (1.0f / 16777216.0f);
    return minstd_uniform(r);
}
static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* multi-draw expression order: 0 = left to right (nvcc build), 1 = right to left (g++ build) */
static inline void draw2(rng_t* r, int order, float* a, float* b) {
    if (order == 0) { *a = U(r); *b = U(r); } else { *b = U(r); *a = U(r); }
}
static inline void draw3(rng_t* r, int order, float* a, float* b, float* c) {
    if (order == 0) { *a = U(r); *b = U(r); *c = U(r); } else { *c = U(r); *b = U(r); *a = U(r); }
}

/* ---------------------------------------------------------------------------------------------- */
/* scene                                                                                          */
/* ---------------------------------------------------------------------------------------------- */
enum { K_LIGHT = 0, K_SPHERE = 1, K_QUAD = 2, K_TRI = 3, K_RECT = 4 };

typedef struct {
    int kind;
    int mat;          /* material index (lights: index into the appended light materials) */
    int light;        /* light index for K_LIGHT */
    int invisible;
    int sphere_light; /* omni / spot light: a sphere (a = center, rad) */
    v3 a, b, c;       /* sphere: a=center, r in rad;  quad/light: a=Q|P, b=u, c=v;  tri: a=v0, b=v0v1, c=v0v2 */
    float rad;
    v3 normal, w;     /* planar */
    float D, area;
    v3 mid;           /* triangle middle_normal */
    int smooth; v3 vn[3];
    float uv[6];      /* triangle: per-vertex texture coordinates (zeros without) */
    float lo[3], hi[3];
    int xf;           /* transform index or -1 (rt::translate / rotate / scale around the primitive) */
    int gid;          /* global object id (one per box) */
    int axis, flip;   /* box face: 0 xy_rect, 1 xz_rect, 2 yz_rect; flip_normals on the low faces */
    float r0, r1, s0, s1, k;   /* box face bounds in its two in-plane axes and its plane */
} prim_t;

/* rt::translate / rt::rotate / rt::scale (primitives/translate.cuh, rotate.cuh, scale.cuh) */
typedef struct { v3 t, s; float inv[3][3], fwd[3][3]; unsigned flags; } xf_t;

typedef struct { int kind; float col[3]; float inv_scale; int even, odd, image; } tex_t;
/* kind MAT_SPOT (4): diffuse_spot_light (materials/diffuse_spot_light.cuh), cone in dir/cos_cutoff/falloff */
enum { MAT_SPOT = 4 };
typedef struct {
    int kind; int tex; float fuzz, ior, intensity; int directional;
    v3 dir; float cos_cutoff, falloff; int invisible;
} mat_t;
typedef struct { float lo[3], hi[3]; int left, right, first, count; } node_t;

typedef struct {
    prim_t* prims; int nprims;
    xf_t* xf; int nxf;
    int* order;           /* BVH leaf order */
    node_t* nodes; int nnodes;
    tex_t* tex; int ntex;
    mat_t* mat; int nmat;
    rtc_image* img; int nimg;
    unsigned char** img_bytes;
    int* lights; int nlights;   /* prim index of each light, in light-list order */
    rtc_camera cam;
    rtc_background bg;
    float* env;
    int any_uv;           /* a mesh has texture coordinates: triangles evaluate them at the hit */
} scene_t;

static void box_grow(float* lo, float* hi, v3 p) {
    float c[3] = {p.x, p.y, p.z};
    for (int k = 0; k < 3; ++k) { if (c[k] < lo[k]) lo[k] = c[k]; if (c[k] > hi[k]) hi[k] = c[k]; }
}

/* quad::quad (quad.cuh:55-67) / directional_light ctor (directional_light.cuh:45-58) */
static void planar_init(prim_t* p) {
    v3 n = vcross(p->b, p->c);
    p->normal = vunit(n);
    p->D = vdot(p->normal, p->a);
    p->w = vdivs(n, vdot(n, n));
    p->area = vlen(n);
}

/* glm::rotate(m, angle, axis) for a coordinate axis (glm/ext/matrix_transform.inl:18-46), float, same
 * operation order; m column-major m[column][row] */
static void glm_rotate_axis(float m[4][4], float angle, int ax) {
    const float c = cosf(angle), sn = sinf(angle);
    float axis[3] = {0.0f, 0.0f, 0.0f}, R[3][3], out[3][4];
    axis[ax] = 1.0f;
    const float temp[3] = {(1.0f - c) * axis[0], (1.0f - c) * axis[1], (1.0f - c) * axis[2]};
    R[0][0] = c + temp[0] * axis[0];
    R[0][1] = temp[0] * axis[1] + sn * axis[2];
    R[0][2] = temp[0] * axis[2] - sn * axis[1];
    R[1][0] = temp[1] * axis[0] - sn * axis[2];
    R[1][1] = c + temp[1] * axis[1];
    R[1][2] = temp[1] * axis[2] + sn * axis[0];
    R[2][0] = temp[2] * axis[0] + sn * axis[1];
    R[2][1] = temp[2] * axis[1] - sn * axis[0];
    R[2][2] = c + temp[2] * axis[2];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 4; ++i) out[j][i] = (m[0][i] * R[j][0] + m[1][i] * R[j][1]) + m[2][i] * R[j][2];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 4; ++i) m[j][i] = out[j][i];
}
/* rt::rotate's matrix: identity rotated about x, y, z by degrees_to_radians(sign * angle) (float M_PI) */
static void rotate_matrix(const float deg[3], float sign, float out[3][3]) {
    float m[4][4];
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i) m[j][i] = i == j ? 1.0f : 0.0f;
    for (int ax = 0; ax < 3; ++ax) glm_rotate_axis(m, (sign * deg[ax]) * PI_F / 180.0f, ax);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) out[j][i] = m[j][i];
}
/* glm mat4 * vec4 for a rotation: (m0_i x + m1_i y) + (m2_i z + 0) */
static v3 rot_apply(const float m[3][3], v3 v) {
    return V((m[0][0] * v.x + m[1][0] * v.y) + (m[2][0] * v.z + 0.0f), (m[0][1] * v.x + m[1][1] * v.y) + (m[2][1] * v.z + 0.0f),
             (m[0][2] * v.x + m[1][2] * v.y) + (m[2][2] * v.z + 0.0f));
}
/* world ray -> object space: scale (o / s, d / s), rotate (inverse matrix), translate (o - t) */
static void xf_to_object(const xf_t* x, v3* o, v3* d) {
    if (x->flags & 4u) { *o = V(o->x / x->s.x, o->y / x->s.y, o->z / x->s.z); *d = V(d->x / x->s.x, d->y / x->s.y, d->z / x->s.z); }
    if (x->flags & 2u) { *o = rot_apply(x->inv, *o); *d = rot_apply(x->inv, *d); }
    if (x->flags & 1u) *o = vsub(*o, x->t);
}
/* hit point / normal -> world: translate (+t), rotate (forward matrix), scale (p * s, unit(n / s)) */
static void xf_to_world(const xf_t* x, v3* p, v3* n) {
    if (x->flags & 1u) *p = vadd(*p, x->t);
    if (x->flags & 2u) { *p = rot_apply(x->fwd, *p); *n = rot_apply(x->fwd, *n); }
    if (x->flags & 4u) { *p = V(p->x * x->s.x, p->y * x->s.y, p->z * x->s.z); *n = vunit(V(n->x / x->s.x, n->y / x->s.y, n->z / x->s.z)); }
}
/* world bounds of an object-space box through x: corners mapped by s * R_inv^T (c + t), in double */
static void xf_box(const xf_t* x, float* lo, float* hi) {
    double L[3] = {INFINITY, INFINITY, INFINITY}, H[3] = {-INFINITY, -INFINITY, -INFINITY}, mag = 0.0, smax = 1.0;
    for (int c = 0; c < 8; ++c) {
        double p[3] = {(c & 1) ? hi[0] : lo[0], (c & 2) ? hi[1] : lo[1], (c & 4) ? hi[2] : lo[2]}, q[3];
        if (x->flags & 1u) { p[0] += x->t.x; p[1] += x->t.y; p[2] += x->t.z; }
        for (int k = 0; k < 3; ++k) if (fabs(p[k]) > mag) mag = fabs(p[k]);
        if (x->flags & 2u) {
            for (int k = 0; k < 3; ++k) q[k] = x->inv[k][0] * p[0] + x->inv[k][1] * p[1] + x->inv[k][2] * p[2];
            for (int k = 0; k < 3; ++k) p[k] = q[k];
        }
        if (x->flags & 4u) { p[0] *= x->s.x; p[1] *= x->s.y; p[2] *= x->s.z; }
        for (int k = 0; k < 3; ++k) { if (p[k] < L[k]) L[k] = p[k]; if (p[k] > H[k]) H[k] = p[k]; }
    }
    if (x->flags & 4u) smax = fmax(fabs(x->s.x), fmax(fabs(x->s.y), fabs(x->s.z)));
    const double e = 4e-6 * mag * smax + 1e-6;
    for (int k = 0; k < 3; ++k) { lo[k] = (float)(L[k] - e); hi[k] = (float)(H[k] + e); }
}

static int cmp_axis;
static const prim_t* cmp_prims;
static int cmp_cent(const void* x, const void* y) {
    const prim_t* a = &cmp_prims[*(const int*)x];
    const prim_t* b = &cmp_prims[*(const int*)y];
    float ca = a->lo[cmp_axis] + a->hi[cmp_axis], cb = b->lo[cmp_axis] + b->hi[cmp_axis];
    return (ca > cb) - (ca < cb);
}

static int build_node(scene_t* s, int first, int count) {
    int id = s->nnodes++;
    node_t* nd = &s->nodes[id];
    for (int k = 0; k < 3; ++k) { nd->lo[k] = FLT_MAX; nd->hi[k] = -FLT_MAX; }
    for (int i = first; i < first + count; ++i) {
        const prim_t* p = &s->prims[s->order[i]];
        for (int k = 0; k < 3; ++k) {
            if (p->lo[k] < nd->lo[k]) nd->lo[k] = p->lo[k];
            if (p->hi[k] > nd->hi[k]) nd->hi[k] = p->hi[k];
        }
    }
    if (count <= 2) { nd->left = nd->right = -1; nd->first = first; nd->count = count; return id; }
    int ax = 0;
    for (int k = 1; k < 3; ++k) if (nd->hi[k] - nd->lo[k] > nd->hi[ax] - nd->lo[ax]) ax = k;
    cmp_axis = ax; cmp_prims = s->prims;
    qsort(s->order + first, count, sizeof(int), cmp_cent);
    int half = count / 2;
    int l = build_node(s, first, half);
    int r = build_node(s, first + half, count - half);
    s->nodes[id].left = l; s->nodes[id].right = r; s->nodes[id].count = 0;
    return id;
}

void* port_scene_create(const rtc_scene_desc* d) {
    scene_t* s = (scene_t*)calloc(1, sizeof(scene_t));
    if (!s || !d) { snprintf(g_err, sizeof g_err, "bad argument"); free(s); return NULL; }
    int ntri = 0;
    for (uint32_t m = 0; m < d->num_meshes; ++m) ntri += (int)d->meshes[m].num_triangles;
    const int n_omni = (int)d->num_omni_lights, n_dir = (int)d->num_dir_lights, n_spot = (int)d->num_spot_lights;
    const int n_lights = n_omni + n_dir + n_spot;   /* light list: omni, directional, spot (gpu.cu:504-523) */
    s->nprims = n_lights + (int)(d->num_spheres + d->num_quads) + 6 * (int)d->num_boxes + ntri;
    s->prims = (prim_t*)calloc((size_t)s->nprims + 1, sizeof(prim_t));
    s->ntex = (int)d->num_textures + n_lights;
    s->tex = (tex_t*)calloc((size_t)s->ntex + 1, sizeof(tex_t));
    s->nmat = (int)d->num_materials + n_lights;
    s->mat = (mat_t*)calloc((size_t)s->nmat + 1, sizeof(mat_t));
    s->nlights = n_lights;
    s->lights = (int*)calloc((size_t)s->nlights + 1, sizeof(int));
    for (uint32_t i = 0; i < d->num_textures; ++i) {
        const rtc_texture* t = &d->textures[i];
        tex_t* o = &s->tex[i];
        o->kind = t->kind; memcpy(o->col, t->color, 12);
        o->inv_scale = t->kind == RTC_TEX_CHECKER ? 1.0f / t->scale : 0.0f;   /* checker_texture.cuh:23 */
        o->even = t->even; o->odd = t->odd; o->image = t->image;
    }
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        const rtc_material* m = &d->materials[i];
        mat_t* o = &s->mat[i];
        o->kind = m->kind; o->tex = m->texture; o->fuzz = m->fuzz < 1.0f ? m->fuzz : 1.0f;   /* metal.cuh:52 */
        o->ior = m->ior; o->intensity = m->intensity; o->directional = m->directional;
    }
    s->nimg = (int)d->num_images;
    s->img = (rtc_image*)calloc((size_t)s->nimg + 1, sizeof(rtc_image));
    for (int i = 0; i < s->nimg; ++i) s->img[i] = d->images[i];
    s->cam = d->camera;
    s->bg = d->background;
    s->nxf = (int)d->num_transforms;
    s->xf = (xf_t*)calloc((size_t)s->nxf + 1, sizeof(xf_t));
    for (int i = 0; i < s->nxf; ++i) {
        const rtc_transform* T = &d->transforms[i];
        xf_t* x = &s->xf[i];
        x->t = Vp(T->translate); x->s = Vp(T->scale); x->flags = T->flags & 7u;
        rotate_matrix(T->rotate, -1.0f, x->inv);
        rotate_matrix(T->rotate, 1.0f, x->fwd);
    }
    for (int i = 0; i < s->nprims; ++i) { s->prims[i].xf = -1; s->prims[i].gid = i; }
    int k = 0;
    /* omni and spot lights: spheres (omni_light.cuh / spot_light.cuh) */
    for (int j = 0; j < n_omni + n_spot; ++j) {
        const int is_spot = j >= n_omni, li = is_spot ? n_omni + n_dir + (j - n_omni) : j;
        const float* pos = is_spot ? d->spot_lights[j - n_omni].position : d->omni_lights[j].position;
        const float radius = is_spot ? d->spot_lights[j - n_omni].radius : d->omni_lights[j].radius;
        const float* col = is_spot ? d->spot_lights[j - n_omni].color : d->omni_lights[j].color;
        const float inten = is_spot ? d->spot_lights[j - n_omni].intensity : d->omni_lights[j].intensity;
        prim_t* p = &s->prims[li];
        p->kind = K_LIGHT; p->light = li; p->sphere_light = 1;
        p->invisible = is_spot ? d->spot_lights[j - n_omni].invisible : d->omni_lights[j].invisible;
        p->a = Vp(pos); p->rad = radius;
        int ti = (int)d->num_textures + li, mi = (int)d->num_materials + li;
        s->tex[ti].kind = RTC_TEX_SOLID; memcpy(s->tex[ti].col, col, 12);
        s->mat[mi].tex = ti; s->mat[mi].intensity = inten;
        if (is_spot) {
            const rtc_spot_light* L = &d->spot_lights[j - n_omni];
            /* diffuse_spot_light(solid(color), pos, dir, cos(degrees_to_radians(cutoff)), falloff, ...) */
            float rad = L->cutoff * PI_F / 180.0f;   /* degrees_to_radians with the float M_PI */
            s->mat[mi].kind = MAT_SPOT; s->mat[mi].directional = 1;
            s->mat[mi].dir = Vp(L->direction); s->mat[mi].cos_cutoff = cosf(rad); s->mat[mi].falloff = L->falloff;
            s->mat[mi].invisible = L->invisible;
        } else {
            /* m_mat = new diffuse_light(m_color, intensity, false, invisible) (omni_light.cuh:16) */
            s->mat[mi].kind = RTC_MAT_DIFFUSE_LIGHT; s->mat[mi].directional = 0;
        }
        p->mat = mi;
        s->lights[li] = li;
        float r = fabsf(radius);
        for (int q = 0; q < 3; ++q) { p->lo[q] = FLT_MAX; p->hi[q] = -FLT_MAX; }
        box_grow(p->lo, p->hi, vsub(p->a, V(r, r, r))); box_grow(p->lo, p->hi, vadd(p->a, V(r, r, r)));
    }
    k = n_omni;
    for (uint32_t i = 0; i < d->num_dir_lights; ++i, ++k) {
        const rtc_dir_light* L = &d->dir_lights[i];
        prim_t* p = &s->prims[k];
        p->kind = K_LIGHT; p->light = k; p->invisible = L->invisible;
        p->a = Vp(L->position); p->b = Vp(L->u); p->c = Vp(L->v);
        planar_init(p);
        int ti = (int)d->num_textures + k, mi = (int)d->num_materials + k;
        s->tex[ti].kind = RTC_TEX_SOLID; memcpy(s->tex[ti].col, L->color, 12);
        /* m_mat = new diffuse_light(m_color, intensity, true, invisible) (directional_light.cuh:48) */
        s->mat[mi].kind = RTC_MAT_DIFFUSE_LIGHT; s->mat[mi].tex = ti; s->mat[mi].intensity = L->intensity;
        s->mat[mi].directional = 1;
        p->mat = mi;
        s->lights[k] = k;
        v3 hu = vscale(0.5f, p->b), hv = vscale(0.5f, p->c);
        for (int q = 0; q < 3; ++q) { p->lo[q] = FLT_MAX; p->hi[q] = -FLT_MAX; }
        box_grow(p->lo, p->hi, vsub(vsub(p->a, hu), hv)); box_grow(p->lo, p->hi, vadd(vsub(p->a, hu), hv));
        box_grow(p->lo, p->hi, vsub(vadd(p->a, hu), hv)); box_grow(p->lo, p->hi, vadd(vadd(p->a, hu), hv));
    }
    k = n_lights;   /* the spot lights sit after the directional ones */
    for (uint32_t i = 0; i < d->num_spheres; ++i, ++k) {
        const rtc_sphere* S = &d->spheres[i];
        prim_t* p = &s->prims[k];
        p->kind = K_SPHERE; p->mat = S->material; p->a = Vp(S->center); p->rad = S->radius;
        float r = fabsf(S->radius);
        for (int q = 0; q < 3; ++q) { p->lo[q] = S->center[q] - r; p->hi[q] = S->center[q] + r; }
        p->xf = d->sphere_transforms ? (int)d->sphere_transforms[i] - 1 : -1;
    }
    for (uint32_t i = 0; i < d->num_quads; ++i, ++k) {
        const rtc_quad* Q = &d->quads[i];
        prim_t* p = &s->prims[k];
        p->kind = K_QUAD; p->mat = Q->material; p->a = Vp(Q->q); p->b = Vp(Q->u); p->c = Vp(Q->v);
        planar_init(p);
        for (int q = 0; q < 3; ++q) { p->lo[q] = FLT_MAX; p->hi[q] = -FLT_MAX; }
        box_grow(p->lo, p->hi, p->a); box_grow(p->lo, p->hi, vadd(p->a, p->b));
        box_grow(p->lo, p->hi, vadd(p->a, p->c)); box_grow(p->lo, p->hi, vadd(vadd(p->a, p->b), p->c));
        p->xf = d->quad_transforms ? (int)d->quad_transforms[i] - 1 : -1;
    }
    /* boxes (box.cuh:40-52): six faces, pmin = center - size / 2, pmax = pmin + size; face order front
     * (z = pmax.z), back (z = pmin.z, flipped), top, bottom (flipped), right, left (flipped) */
    const int box_gid0 = k;
    for (uint32_t i = 0; i < d->num_boxes; ++i) {
        const rtc_box* B = &d->boxes[i];
        float lo[3], hi[3];
        for (int q = 0; q < 3; ++q) { lo[q] = B->center[q] - (B->size[q] / 2.0f); hi[q] = lo[q] + B->size[q]; }
        for (int f = 0; f < 6; ++f, ++k) {
            prim_t* p = &s->prims[k];
            const int axis = f / 2, low = f & 1;
            const int a = axis == 2 ? 1 : 0, b = axis == 0 ? 1 : 2, n = axis == 0 ? 2 : axis == 1 ? 1 : 0;
            p->kind = K_RECT; p->mat = B->material; p->axis = axis; p->flip = low;
            p->r0 = lo[a]; p->r1 = hi[a]; p->s0 = lo[b]; p->s1 = hi[b]; p->k = low ? lo[n] : hi[n];
            p->xf = (int)B->transform - 1;
            p->gid = box_gid0 + (int)i;
            for (int q = 0; q < 3; ++q) { p->lo[q] = lo[q]; p->hi[q] = hi[q]; }
            p->lo[n] = p->hi[n] = p->k;
        }
    }
    const int tri_gid_shift = 5 * (int)d->num_boxes;   /* one id per box, not per face */
    for (uint32_t m = 0; m < d->num_meshes; ++m) {
        const rtc_mesh* M = &d->meshes[m];
        for (uint32_t f = 0; f < M->num_triangles; ++f, ++k) {
            prim_t* p = &s->prims[k];
            uint32_t ia = M->indices[3 * f], ib = M->indices[3 * f + 1], ic = M->indices[3 * f + 2];
            v3 v0 = Vp(M->vertices + 3 * ia), v1 = Vp(M->vertices + 3 * ib), v2 = Vp(M->vertices + 3 * ic);
            p->kind = K_TRI; p->mat = M->material;
            /* triangle::triangle (triangle.cuh:87-123) */
            p->a = v0; p->b = vsub(v1, v0); p->c = vsub(v2, v0);
            p->mid = vunit(vcross(vsub(v0, v1), vsub(v0, v2)));
            p->smooth = M->smooth && M->normals;
            if (p->smooth) {
                p->vn[0] = vunit(Vp(M->normals + 3 * ia)); p->vn[1] = vunit(Vp(M->normals + 3 * ib));
                p->vn[2] = vunit(Vp(M->normals + 3 * ic));
            }
            if (M->uvs) {
                const uint32_t vi[3] = {ia, ib, ic};
                for (int q = 0; q < 3; ++q) { p->uv[2 * q] = M->uvs[2 * vi[q]]; p->uv[2 * q + 1] = M->uvs[2 * vi[q] + 1]; }
                s->any_uv = 1;
            }
            for (int q = 0; q < 3; ++q) { p->lo[q] = FLT_MAX; p->hi[q] = -FLT_MAX; }
            box_grow(p->lo, p->hi, v0); box_grow(p->lo, p->hi, v1); box_grow(p->lo, p->hi, v2);
            p->xf = d->mesh_transforms ? (int)d->mesh_transforms[m] - 1 : -1;
            p->gid = k - tri_gid_shift;
        }
    }
    for (int i = 0; i < s->nprims; ++i)
        if (s->prims[i].xf >= 0) xf_box(&s->xf[s->prims[i].xf], s->prims[i].lo, s->prims[i].hi);
    for (int i = 0; i < s->nprims; ++i)   /* conservative padding */
        for (int q = 0; q < 3; ++q) {
            float e = 1e-4f * (fabsf(s->prims[i].lo[q]) + fabsf(s->prims[i].hi[q])) + 1e-5f;
            s->prims[i].lo[q] -= e; s->prims[i].hi[q] += e;
        }
    s->order = (int*)malloc(sizeof(int) * ((size_t)s->nprims + 1));
    for (int i = 0; i < s->nprims; ++i) s->order[i] = i;
    s->nodes = (node_t*)calloc(2 * (size_t)s->nprims + 2, sizeof(node_t));
    if (s->nprims > 0) build_node(s, 0, s->nprims);
    if (d->background.kind == RTC_BG_ENV_MAP) s->env = (float*)d->background.env_rgb;   /* caller keeps it alive */
    return s;
}

void port_scene_destroy(void* p) {
    scene_t* s = (scene_t*)p;
    if (!s) return;
    free(s->prims); free(s->order); free(s->nodes); free(s->tex); free(s->mat); free(s->img); free(s->lights); free(s->xf);
    free(s);
}

/* ---------------------------------------------------------------------------------------------- */
/* intersection                                                                                   */
/* ---------------------------------------------------------------------------------------------- */
typedef struct { float t; int prim; v3 p, n; float u, v; int front, mat; } hit_t;

/* hit_record::set_face_normal (hit_record.cuh:34-38) */
static inline void face(hit_t* h, v3 dir, v3 outward) {
    h->front = vdot(dir, outward) < 0.0f;
    h->n = h->front ? outward : vneg(outward);
}

/* sphere::hit (sphere.cuh:111-135) */
static int sphere_t(const prim_t* p, v3 o, v3 d, float tmin, float tmax, float* t) {
    v3 oc = vsub(o, p->a);
    float a = vlensq(d);
    float half_b = oc.x * d.x + oc.y * d.y + oc.z * d.z;
    float c = vlensq(oc) - p->rad * p->rad;
    float disc = half_b * half_b - a * c;
    if (disc < 0) return 0;
    float sq = sqrtf(disc);
    float root = (-half_b - sq) / a;
    if (!(tmin < root && root < tmax)) {
        root = (-half_b + sq) / a;
        if (!(tmin < root && root < tmax)) return 0;
    }
    *t = root;
    return 1;
}

/* Clean mode: the same quadratic in double (the float form cancels catastrophically for large
 * spheres; the clean kernels do the same). */
static int sphere_t_exact(const prim_t* p, v3 o, v3 d, float tmin, float tmax, float* t) {
    double ox = (double)o.x - (double)p->a.x, oy = (double)o.y - (double)p->a.y, oz = (double)o.z - (double)p->a.z;
    double dx = d.x, dy = d.y, dz = d.z;
    double a = dx * dx + dy * dy + dz * dz;
    double hb = ox * dx + oy * dy + oz * dz;
    double c = ox * ox + oy * oy + oz * oz - (double)p->rad * (double)p->rad;
    double disc = hb * hb - a * c;
    if (disc < 0.0) return 0;
    double sq = sqrt(disc);
    double root = (-hb - sq) / a;
    if (!((double)tmin < root && root < (double)tmax)) {
        root = (-hb + sq) / a;
        if (!((double)tmin < root && root < (double)tmax)) return 0;
    }
    *t = (float)root;
    return 1;
}

/* quad::hit (quad.cuh:100-133) and directional_light::hit (directional_light.cuh:76-120) */
static int planar_t(const prim_t* p, v3 o, v3 d, float tmin, float tmax, int centred, float* t, float* al, float* be) {
    float denom = vdot(p->normal, d);
    if (fabs(denom) < 1e-8) return 0;
    float tt = (p->D - vdot(p->normal, o)) / denom;
    if (!(tmin <= tt && tt <= tmax)) return 0;
    v3 ip = vat(o, d, tt);
    v3 pl = vsub(ip, p->a);
    float a = vdot(p->w, vcross(pl, p->c));
    float b = vdot(p->w, vcross(p->b, pl));
    if (centred) { if ((a < -0.5) || (0.5 < a) || (b < -0.5) || (0.5 < b)) return 0; }
    else { if ((a < 0) || (1 < a) || (b < 0) || (1 < b)) return 0; }
    *t = tt; *al = a; *be = b;
    return 1;
}

/* triangle::hit (triangle.cuh:130-160) */
static int tri_t(const prim_t* p, v3 o, v3 d, float tmin, float tmax, float* t, float* bu, float* bv) {
    v3 pv = vcross(d, p->c);
    float det = vdot(p->b, pv);
    if (fabsf(det) < 0.000001f) return 0;
    float inv_det = 1.0f / det;
    v3 tv = vsub(o, p->a);
    float u = vdot(tv, pv) * inv_det;
    if (u < 0 || u > 1) return 0;
    v3 qv = vcross(tv, p->b);
    float v = vdot(d, qv) * inv_det;
    if (v < 0 || u + v > 1) return 0;
    float tt = vdot(p->c, qv) * inv_det;
    if (tt < tmin || tt > tmax) return 0;
    *t = tt; *bu = u; *bv = v;
    return 1;
}

/* xy_rect / xz_rect / yz_rect::hit (aarect.cuh): inclusive interval and bounds */
static int rect_t(const prim_t* p, v3 o, v3 d, float tmin, float tmax, float* t, float* al, float* be) {
    const float oa = p->axis == 0 ? o.z : p->axis == 1 ? o.y : o.x, da = p->axis == 0 ? d.z : p->axis == 1 ? d.y : d.x;
    const float tt = (p->k - oa) / da;
    if (tt < tmin || tt > tmax) return 0;
    const float o0 = p->axis == 2 ? o.y : o.x, d0 = p->axis == 2 ? d.y : d.x;
    const float o1 = p->axis == 0 ? o.y : o.z, d1 = p->axis == 0 ? d.y : d.z;
    const float a = o0 + tt * d0, b = o1 + tt * d1;
    if (a < p->r0 || a > p->r1 || b < p->s0 || b > p->s1) return 0;
    *t = tt; *al = a; *be = b;
    return 1;
}

static int prim_t_test_xf(const scene_t* s, const prim_t* p, v3 o, v3 d, float tmin, float tmax, int hide, int exact,
                          float* t);
static int prim_t_test(const prim_t* p, v3 o, v3 d, float tmin, float tmax, int hide, int exact, float* t) {
    float a, b;
    switch (p->kind) {
    case K_RECT: return rect_t(p, o, d, tmin, tmax, t, &a, &b);
    case K_SPHERE: return exact ? sphere_t_exact(p, o, d, tmin, tmax, t) : sphere_t(p, o, d, tmin, tmax, t);
    case K_QUAD: return planar_t(p, o, d, tmin, tmax, 0, t, &a, &b);
    case K_LIGHT:
        if (p->sphere_light) {   /* omni_light::hit (omni_light.cuh:55-83) */
            if (!(exact ? sphere_t_exact(p, o, d, tmin, tmax, t) : sphere_t(p, o, d, tmin, tmax, t))) return 0;
        } else if (!planar_t(p, o, d, tmin, tmax, 1, t, &a, &b)) {
            return 0;
        }
        return !(p->invisible && hide);   /* directional_light.cuh:106, omni_light.cuh:76-80 */
    default: return tri_t(p, o, d, tmin, tmax, t, &a, &b);
    }
}
static int prim_t_test_xf(const scene_t* s, const prim_t* p, v3 o, v3 d, float tmin, float tmax, int hide, int exact,
                          float* t) {
    if (p->xf >= 0) xf_to_object(&s->xf[p->xf], &o, &d);
    return prim_t_test(p, o, d, tmin, tmax, hide, exact, t);
}

/* aabb::hit semantics (aabb.cuh:141-166) on the port's own (padded) boxes */
static int box_hit(const node_t* n, v3 o, v3 d, float tmin, float tmax) {
    const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    for (int a = 0; a < 3; ++a) {
        float invD = 1 / dd[a];
        float t0 = (n->lo[a] - oo[a]) * invD, t1 = (n->hi[a] - oo[a]) * invD;
        if (invD < 0) { float tmp = t0; t0 = t1; t1 = tmp; }
        if (t0 > tmin) tmin = t0;
        if (t1 < tmax) tmax = t1;
        if (tmax < tmin) return 0;
    }
    return 1;
}

/* exact: clean mode's double-precision sphere test */
static int closest(const scene_t* s, v3 o, v3 d, float tmin, float tmax, int hide, int exact, float* tout, int* pout) {
    int stack[128], sp = 0, best = -1;
    float best_t = tmax;
    if (s->nprims == 0) return 0;
    stack[sp++] = 0;
    while (sp) {
        const node_t* n = &s->nodes[stack[--sp]];
        if (!box_hit(n, o, d, tmin, best_t)) continue;
        if (n->left < 0) {
            for (int i = n->first; i < n->first + n->count; ++i) {
                float t;
                if (prim_t_test_xf(s, &s->prims[s->order[i]], o, d, tmin, best_t, hide, exact, &t)) { best_t = t; best = s->order[i]; }
            }
        } else {
            if (sp + 2 > 128) return 0;
            stack[sp++] = n->right;
            stack[sp++] = n->left;
        }
    }
    *tout = best_t; *pout = best;
    return best >= 0;
}

/* the rest of each hit() for the winner */
static void finalize(const scene_t* s, int pi, float t, v3 o, v3 d, hit_t* h) {
    const prim_t* p = &s->prims[pi];
    h->t = t; h->prim = pi; h->mat = p->mat;
    if (p->xf >= 0) xf_to_object(&s->xf[p->xf], &o, &d);
    if (p->kind == K_RECT) {
        /* aarect hit(): r.at(t), the axis normal (flip_normals negates it), front_face stays true, uv by
         * get_xy/xz/yz_rect_uv with the default mapping */
        const float o0 = p->axis == 2 ? o.y : o.x, d0 = p->axis == 2 ? d.y : d.x;
        const float o1 = p->axis == 0 ? o.y : o.z, d1 = p->axis == 0 ? d.y : d.z;
        const float a = o0 + t * d0, b = o1 + t * d1;
        float su = (a - p->r0) / (p->r1 - p->r0), sv = (b - p->s0) / (p->s1 - p->s0);
        su = fmodf(su * 1.0f, 1.0f); sv = fmodf(sv * 1.0f, 1.0f);
        h->u = 1.0f * su + 0.0f; h->v = 1.0f * sv + 0.0f;
        h->p = vat(o, d, t);
        const float sg = p->flip ? -1.0f : 1.0f;
        h->n = p->axis == 0 ? V(0.0f, 0.0f, sg) : p->axis == 1 ? V(0.0f, sg, 0.0f) : V(sg, 0.0f, 0.0f);
        h->front = 1;
    } else if (p->kind == K_SPHERE) {
        h->p = vat(o, d, t);
        v3 outward = vdivs(vsub(h->p, p->a), p->rad);
        face(h, d, outward);
        /* get_sphere_uv (uvmapping.cuh:204-228), default mapping */
        float theta = f_acos(-outward.y);
        float phi = f_atan2(-outward.z, outward.x) + PI_F;
        float sc = phi / (2 * PI_F), tc = theta / PI_F;
        sc = fmodf(sc * 1.0f, 1.0f); tc = fmodf(tc * 1.0f, 1.0f);
        h->u = 1.0f * sc + 0.0f; h->v = 1.0f * tc + 0.0f;
    } else if (p->kind == K_LIGHT && p->sphere_light) {
        h->p = vat(o, d, t);
        face(h, d, vdivs(vsub(h->p, p->a), p->rad));
        h->u = 0.0f; h->v = 0.0f;   /* solid texture: uv unused */
    } else if (p->kind == K_QUAD || p->kind == K_LIGHT) {
        v3 ip = vat(o, d, t), pl = vsub(ip, p->a);
        float a = vdot(p->w, vcross(pl, p->c)), b = vdot(p->w, vcross(p->b, pl));
        h->p = ip;
        face(h, d, p->normal);
        if (p->kind == K_QUAD) { h->u = a; h->v = b; } else { h->u = a + 0.5f; h->v = b + 0.5f; }
    } else {
        h->p = vat(o, d, t);
        v3 normal = p->mid;
        if (p->smooth) {
            v3 pv = vcross(d, p->c);
            float inv_det = 1.0f / vdot(p->b, pv);
            v3 tv = vsub(o, p->a);
            float bu = vdot(tv, pv) * inv_det;
            float bv = vdot(d, vcross(tv, p->b)) * inv_det;
            float bc = 1 - bu - bv;
            normal = vadd(vadd(vscale(bu, p->vn[1]), vscale(bv, p->vn[2])), vscale(bc, p->vn[0]));
        }
        face(h, d, normal);
        if (s->any_uv) {
            /* get_triangle_uv (uvmapping.cuh:415-429) at this hit's point: get_barycenter (math_utils.cuh:
               73-86), then calculateTextureCoordinate with its wrap (uvmapping.cuh:435-447); the reference
               passes the record's previous hit point (triangle.cuh:162), here the hit's own */
            v3 p2 = vsub(h->p, p->a);
            float d00 = vdot(p->b, p->b), d01 = vdot(p->b, p->c), d11 = vdot(p->c, p->c);
            float d20 = vdot(p2, p->b), d21 = vdot(p2, p->c);
            float denom = d00 * d11 - d01 * d01;
            float bv = (d11 * d20 - d01 * d21) / denom;
            float bw = (d00 * d21 - d01 * d20) / denom;
            float bu = 1.0f - bv - bw;
            float tu = bu * p->uv[0] + bv * p->uv[2] + (1.0f - bu - bv) * p->uv[4];
            float tv = bu * p->uv[1] + bv * p->uv[3] + (1.0f - bu - bv) * p->uv[5];
            tu = fmodf(tu, 1.0f); tv = fmodf(tv, 1.0f);
            if (tu < 0.0f) tu += 1.0f;
            if (tv < 0.0f) tv += 1.0f;
            h->u = tu; h->v = tv;
        } else {
            h->u = 0.0f; h->v = 0.0f;   /* get_triangle_uv over all-zero vertex uvs */
        }
    }
    if (p->xf >= 0) xf_to_world(&s->xf[p->xf], &h->p, &h->n);
}

/* ---------------------------------------------------------------------------------------------- */
/* shading                                                                                        */
/* ---------------------------------------------------------------------------------------------- */
typedef struct { float r, g, b; } rgb_t;

/* texture::value: solid / checker / image (solid_color_texture.cuh:34, checker_texture.cuh:33-41,
   image_texture.cuh:54-70, bitmap_image.cuh:74-91) */
static rgb_t tex_value(const scene_t* s, int ti, float u, float v, v3 p) {
    for (int guard = 0; guard < 8 && ti >= 0 && ti < s->ntex; ++guard) {
        const tex_t* t = &s->tex[ti];
        if (t->kind == RTC_TEX_SOLID) { rgb_t c = {t->col[0], t->col[1], t->col[2]}; return c; }
        if (t->kind == RTC_TEX_CHECKER) {
            int xi = (int)floorf(t->inv_scale * p.x), yi = (int)floorf(t->inv_scale * p.y), zi = (int)floorf(t->inv_scale * p.z);
            ti = ((xi + yi + zi) % 2 == 0) ? t->even : t->odd;
            continue;
        }
        const rtc_image* im = &s->img[t->image];
        if (im->height <= 0) { rgb_t c = {0, 1, 1}; return c; }
        float uu = u < 0 ? 0 : (u > 1 ? 1 : u);
        float vc = v < 0 ? 0 : (v > 1 ? 1 : v);
        float vv = 1.0f - vc;
        int i = (int)(uu * im->width), j = (int)(vv * im->height);
        i = i < 0 ? 0 : (i < im->width ? i : im->width - 1);
        j = j < 0 ? 0 : (j < im->height ? j : im->height - 1);
        const unsigned char* px = im->rgb + (size_t)j * im->width * 3 + (size_t)i * 3;
        float cs = 1.0f / 255.0f;
        rgb_t c = {cs * px[0], cs * px[1], cs * px[2]};
        return c;
    }
    rgb_t z = {0, 0, 0};
    return z;
}

static rgb_t background(const scene_t* s, v3 dir) {
    const rtc_background* B = &s->bg;
    rgb_t c;
    if (B->kind == RTC_BG_CONSTANT) { c.r = B->color[0]; c.g = B->color[1]; c.b = B->color[2]; return c; }
    v3 ud = vunit(dir);
    if (B->kind == RTC_BG_SKY_GRADIENT) {
        float a = 0.5f * (ud.y + 1.0f), b = 1.0f - a;
        c.r = b * B->color[0] + a * B->top[0]; c.g = b * B->color[1] + a * B->top[1]; c.b = b * B->color[2] + a * B->top[2];
        return c;
    }
    double theta = acos((double)-ud.y), phi = atan2((double)-ud.z, (double)ud.x) + 3.14159265358979323846;
    double uu = phi / (2.0 * 3.14159265358979323846), vv = theta / 3.14159265358979323846;
    int W = B->env_width, H = B->env_height;
    int x = (int)(uu * W); x = x < 0 ? 0 : (x >= W ? W - 1 : x);
    int y = (int)((1.0 - vv) * H); y = y < 0 ? 0 : (y >= H ? H - 1 : y);
    const float* px = s->env + 3 * ((size_t)y * W + x);
    c.r = px[0]; c.g = px[1]; c.b = px[2];
    return c;
}

/* directional_light::pdf_value (directional_light.cuh:147-158) */
static float light_pdf(const scene_t* s, int li, v3 o, v3 v) {
    const prim_t* p = &s->prims[s->lights[li]];
    float t, a, b;
    if (p->sphere_light) {   /* omni_light::pdf_value (omni_light.cuh:104-115) */
        if (!sphere_t(p, o, v, 0.00001f, INFINITY, &t)) return 0;
        float ctm = sqrtf(1 - p->rad * p->rad / vlensq(vsub(p->a, o)));
        float solid_angle = 2 * PI_F * (1 - ctm);   /* M_PI is a float literal (misc/constants.cuh:35) */
        return 1.0f / solid_angle;
    }
    if (!planar_t(p, o, v, 0.00001f, INFINITY, 1, &t, &a, &b)) return 0;
    v3 nrm = vdot(v, p->normal) < 0.0f ? p->normal : vneg(p->normal);
    float distance_squared = t * t * vlensq(v);
    float cosine = fabsf(vdot(v, nrm) / vlen(v));
    return distance_squared / (cosine * p->area);
}

typedef struct { v3 u, v, w; } onb_t;
static onb_t build_from_w(v3 n) {   /* onb::build_from_w (onb.cuh:122-128) */
    onb_t b;
    b.w = vunit(n);
    v3 a = (fabsf(b.w.x) > 0.9f) ? V(0, 1, 0) : V(1, 0, 0);
    b.v = vunit(vcross(b.w, a));
    b.u = vcross(b.w, b.v);
    return b;
}
static v3 onb_local(const onb_t* b, v3 a) { return vadd(vadd(vscale(a.x, b->u), vscale(a.y, b->v)), vscale(a.z, b->w)); }

/* Clean mode: scattered rays start from a point offset along the normal of the side they leave from,
   Waechter & Binder, "A Fast and Robust Method for Avoiding Self-Intersection", Ray Tracing Gems
   (2019), ch. 6.  Compat mode starts them at the hit point (the reference's behaviour). */
static inline float offset_coord(float p, float n) {
    const float kOrigin = 1.0f / 32.0f, kFloatScale = 1.0f / 65536.0f, kIntScale = 256.0f;
    int of = (int)(kIntScale * n);
    int32_t bits;
    memcpy(&bits, &p, 4);
    bits += (p < 0.0f ? -of : of);
    float pi;
    memcpy(&pi, &bits, 4);
    return fabsf(p) < kOrigin ? p + kFloatScale * n : pi;
}
static inline v3 scatter_origin(int clean, v3 p, v3 n, v3 dir) {
    if (!clean) return p;
    v3 side = vdot(dir, n) < 0.0f ? vneg(n) : n;
    return V(offset_coord(p.x, side.x), offset_coord(p.y, side.y), offset_coord(p.z, side.z));
}

/* omni_light::random (omni_light.cuh:117-124) with random_to_sphere (gpu_randomizer.cuh:82-93): the
   direction toward a sphere light of centre c and radius r from o (two draws) */
static v3 sphere_light_random(v3 c, float r, v3 o, rng_t* rng) {
    v3 dl = vsub(c, o);
    float dsq = vlensq(dl);
    onb_t lb = build_from_w(dl);
    float r1 = U(rng), r2 = U(rng);
    float z = 1 + r2 * (sqrtf(1 - r * r / dsq) - 1);
    float phi = 2 * PI_F * r1;   /* float M_PI (misc/constants.cuh:35) */
    float x = f_cos(phi) * sqrtf(1 - z * z), y = f_sin(phi) * sqrtf(1 - z * z);
    return onb_local(&lb, V(x, y, z));
}

/* the same sampler for the known-answer test: light (0.3,-0.2,0.1), radius 0.5, seen from (1.3,0.7,-2.1) */
int port_sphere_light_draws(uint32_t seed, int64_t n, float* out) {
    rng_t rng; minstd_seed(&rng, seed);
    for (int64_t k = 0; k < n; ++k) {
        v3 p = sphere_light_random(V(0.3f, -0.2f, 0.1f), 0.5f, V(1.3f, 0.7f, -2.1f), &rng);
        out[3 * k] = p.x; out[3 * k + 1] = p.y; out[3 * k + 2] = p.z;
    }
    return 0;
}

/* camera::ray_color (camera.cuh:149-264) for one sample; returns radiance, counts closest-hit calls */
static rgb_t ray_color(const scene_t* s, v3 o, v3 d, int max_depth, rng_t* rng, int order, int clean, uint64_t* rays) {
    rgb_t res = {0, 0, 0}, att = {1, 1, 1};
    for (int depth = max_depth; depth > 0; --depth) {
        int hide = depth == max_depth;
        float t; int pi;
        (*rays)++;
        if (!closest(s, o, d, 0.00001f, FLT_MAX, hide, clean, &t, &pi)) {
            rgb_t bg = background(s, d);
            res.r += att.r * bg.r; res.g += att.g * bg.g; res.b += att.b * bg.b;
            break;
        }
        hit_t h;
        finalize(s, pi, t, o, d, &h);
        const mat_t* m = &s->mat[h.mat];
        rgb_t em = {0, 0, 0};
        int alpha0 = 0;
        if (m->kind == RTC_MAT_DIFFUSE_LIGHT) {   /* diffuse_light::emitted (diffuse_light.cuh:45-67) */
            if (m->directional && !h.front) alpha0 = 1;
            else { rgb_t tv = tex_value(s, m->tex, h.u, h.v, h.p); em.r = tv.r * m->intensity; em.g = tv.g * m->intensity; em.b = tv.b * m->intensity; }
        } else if (m->kind == MAT_SPOT) {   /* diffuse_spot_light::emitted (diffuse_spot_light.cuh:33-49) */
            if (!h.front) {
                alpha0 = 1;
                if (!m->invisible) { em.r = em.g = em.b = 1.0f; }   /* color(1,1,1,0) */
            } else {
                float cos_theta = vdot(vunit(d), vunit(m->dir));
                if (cos_theta < m->cos_cutoff) {
                    em.r = em.g = em.b = 1.0f;
                } else {
                    float k2 = m->intensity * f_pow(cos_theta, m->falloff);
                    rgb_t tv = tex_value(s, m->tex, h.u, h.v, h.p);
                    em.r = tv.r * k2; em.g = tv.g * k2; em.b = tv.b * k2;
                }
            }
        }
        if (alpha0) {   /* invisible re-hit (camera.cuh:177-183) */
            float t2; int p2;
            (*rays)++;
            if (closest(s, o, d, h.t + 0.001f, FLT_MAX, hide, clean, &t2, &p2)) { finalize(s, p2, t2, o, d, &h); m = &s->mat[h.mat]; }
        }
        if (m->kind == RTC_MAT_DIFFUSE_LIGHT || m->kind == MAT_SPOT) {
            res.r += att.r * em.r; res.g += att.g * em.g; res.b += att.b * em.b;
            break;
        }
        res.r += att.r * em.r; res.g += att.g * em.g; res.b += att.b * em.b;
        if (m->kind == RTC_MAT_METAL) {   /* metal::scatter (metal.cuh:57-64) */
            rgb_t a = tex_value(s, m->tex, h.u, h.v, h.p);
            v3 refl = vreflect(vunit(d), h.n);
            v3 p;
            do {   /* random_in_unit_sphere (gpu_randomizer.cuh:70-76) */
                float x, y, z;
                draw3(rng, order, &x, &y, &z);
                p = V(2.0f * x - 1.0f, 2.0f * y - 1.0f, 2.0f * z - 1.0f);
            } while (p.x * p.x + p.y * p.y + p.z * p.z >= 1.0f);
            d = vadd(refl, vscale(m->fuzz, p));
            o = scatter_origin(clean, h.p, h.n, d);
            att.r *= a.r; att.g *= a.g; att.b *= a.b;
            continue;
        }
        if (m->kind == RTC_MAT_DIELECTRIC) {   /* dielectric::scatter (dielectric.cuh:32-63) */
            float ratio = h.front ? (1.0f / m->ior) : m->ior;
            v3 ud = vunit(d);
            float ct = vdot(vneg(ud), h.n);
            float cos_theta = ct < 1.0f ? ct : 1.0f;
            float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
            int reflect = ratio * sin_theta > 1.0;
            if (!reflect) {
                float r0 = (1 - ratio) / (1 + ratio);
                r0 = r0 * r0;
                float refl = r0 + (1 - r0) * (float)(pow((1 - cos_theta), 5));
                reflect = refl > U(rng);
            }
            d = reflect ? vreflect(ud, h.n) : vrefract(ud, h.n, ratio);
            o = scatter_origin(clean, h.p, h.n, d);
            continue;
        }
        /* lambertian (lambertian.cuh:63-143) + mixture_pdf(hittable_pdf(lights), cosine_pdf) */
        rgb_t a = tex_value(s, m->tex, h.u, h.v, h.p);
        onb_t b = build_from_w(h.n);
        v3 dir;
        float pdf_val;
        int mixture = !clean || s->nlights > 0;
        if (mixture && U(rng) < 0.5f) {
            if (s->nlights == 0) dir = V(0, 0, 0);
            else {
                if (s->nlights > 1) (void)U(rng);   /* get_int(rng, 0, n-1) == 0 */
                const prim_t* L = &s->prims[s->lights[0]];
                if (L->sphere_light) {
                    dir = sphere_light_random(L->a, L->rad, h.p, rng);
                } else {
                    float ru, rv;
                    draw2(rng, order, &ru, &rv);
                    v3 pp = vadd(vadd(L->a, vscale(ru - 0.5f, L->b)), vscale(rv - 0.5f, L->c));
                    dir = vsub(pp, h.p);
                }
            }
        } else {
            float r1 = U(rng), r2 = U(rng);   /* random_cosine_direction (gpu_randomizer.cuh:121-133) */
            float phi = 6.28318530718f * r1;
            float z = sqrtf(1 - r2), r2s = sqrtf(r2);
            dir = onb_local(&b, V(f_cos(phi) * r2s, f_sin(phi) * r2s, z));
        }
        float cosv = vdot(vunit(dir), b.w) / PI_F;
        float cpdf = 0.0f > cosv ? 0.0f : cosv;
        if (mixture) {
            float weight = 1.0f / (float)s->nlights, sum = 0.0f;
            for (int li = 0; li < s->nlights; ++li) sum += weight * light_pdf(s, li, h.p, dir);
            pdf_val = 0.5f * sum + (1.0f - 0.5f) * cpdf;
        } else {
            pdf_val = cpdf;
        }
        float cth = vdot(h.n, vunit(dir));
        float spdf = cth < 0 ? 0.0f : cth / PI_F;
        float rcp = 1 / pdf_val;
        att.r *= rcp * (a.r * spdf); att.g *= rcp * (a.g * spdf); att.b *= rcp * (a.b * spdf);
        o = scatter_origin(clean, h.p, h.n, dir);
        d = dir;
    }
    return res;
}

/* ---------------------------------------------------------------------------------------------- */
/* render loop (render kernel, gpu.cu:761-790)                                                    */
/* ---------------------------------------------------------------------------------------------- */
typedef struct {
    v3 origin, llc, horizontal, vertical, u, v;
    float lens_radius;
} cam_t;

/* perspective_camera::initialize (perspective_camera.cuh:41-108) */
static cam_t make_cam(const rtc_camera* C) {
    cam_t c;
    float theta = C->vfov * PI_F / 180.0f;
    float half_height = tanf(theta / 2);
    v3 w = vunit(vsub(Vp(C->look_from), Vp(C->look_at)));
    v3 u = vunit(vcross(Vp(C->up), w));
    v3 v = vcross(w, u);
    float half_width = C->aspect * half_height, f = C->focus;
    c.origin = Vp(C->look_from);
    c.llc = vsub(vsub(vsub(c.origin, vscale(half_width * f, u)), vscale(half_height * f, v)), vscale(f, w));
    c.horizontal = vscale(2 * half_width * f, u);
    c.vertical = vscale(2 * half_height * f, v);
    c.u = u; c.v = v;
    c.lens_radius = C->aperture / 2;
    return c;
}

typedef struct {
    const scene_t* s; const rtc_render_params* p; const int64_t* pix; int64_t n; float* out;
    cam_t cam; int sq; volatile int64_t next; uint64_t rays; pthread_mutex_t mu;
} job_t;

static void render_one(job_t* J, int64_t q, uint64_t* rays) {
    const rtc_render_params* P = J->p;
    int64_t pixel_index = J->pix[q];
    int i = (int)(pixel_index % P->width), j = (int)(pixel_index / P->width);
    float pr = 0, pg = 0, pb = 0;
    const cam_t* c = &J->cam;
    int clean = P->mode == RTC_MODE_CLEAN, order = clean ? 0 : P->draw_order;
    rng_t rng;
    memset(&rng, 0, sizeof rng);
    int nsamp = clean ? P->spp : J->sq * J->sq;
    if (!clean) minstd_seed(&rng, P->seed + (uint32_t)pixel_index);
    for (int sidx = 0; sidx < nsamp; ++sidx) {
        float u, v;
        if (clean) {
            pcg_seed(&rng, mix64(((uint64_t)P->seed << 32) ^ (uint64_t)pixel_index), (uint64_t)sidx);
            float ju = U(&rng), jv = U(&rng);
            u = ((float)i + ju) / (float)P->width;
            v = ((float)j + jv) / (float)P->height;
        } else {
            int s_j = sidx / J->sq, s_i = sidx % J->sq;
            float ur = U(&rng);
            u = (i + (s_i + ur) / J->sq) / (float)P->width;
            v = (j + (s_j + ur) / J->sq) / (float)P->height;
        }
        /* perspective_camera::get_ray (perspective_camera.cuh:112-117) */
        v3 p;
        do {
            float a, b;
            draw2(&rng, order, &a, &b);
            p = V(2.0f * a - 1.0f, 2.0f * b - 1.0f, 2.0f * 0.0f - 0.0f);
        } while (vdot(p, p) >= 1.0f);
        v3 rd = vscale(c->lens_radius, p);
        v3 offset = vadd(V(c->u.x * rd.x, c->u.y * rd.x, c->u.z * rd.x), V(c->v.x * rd.y, c->v.y * rd.y, c->v.z * rd.y));
        (void)(0.0f + U(&rng) * (1.0f - 0.0f));   /* time sample */
        v3 o = vadd(c->origin, offset);
        v3 d = vsub(vsub(vadd(vadd(c->llc, vscale(u, c->horizontal)), vscale(v, c->vertical)), c->origin), offset);
        rgb_t col = ray_color(J->s, o, d, P->max_depth, &rng, order, clean, rays);
        if (clean && !(isfinite(col.r) && isfinite(col.g) && isfinite(col.b))) continue;
        pr += col.r; pg += col.g; pb += col.b;
    }
    J->out[4 * q] = pr; J->out[4 * q + 1] = pg; J->out[4 * q + 2] = pb; J->out[4 * q + 3] = 1.0f;
}

static void* worker(void* arg) {
    job_t* J = (job_t*)arg;
    uint64_t rays = 0;
    for (;;) {
        int64_t b = __atomic_fetch_add(&J->next, 16, __ATOMIC_RELAXED);
        if (b >= J->n) break;
        int64_t e = b + 16 < J->n ? b + 16 : J->n;
        for (int64_t q = b; q < e; ++q) render_one(J, q, &rays);
    }
    __atomic_fetch_add(&J->rays, rays, __ATOMIC_RELAXED);
    return NULL;
}

int port_render_pixels(void* sp, const rtc_render_params* p, const int64_t* pix, int64_t n, float* out,
                       uint64_t* rays_out, int threads) {
    scene_t* s = (scene_t*)sp;
    if (!s || !p || !out || (n > 0 && !pix)) { snprintf(g_err, sizeof g_err, "bad argument"); return 1; }
    job_t J;
    memset(&J, 0, sizeof J);
    J.s = s; J.p = p; J.pix = pix; J.n = n; J.out = out;
    J.cam = make_cam(&s->cam);
    J.sq = (int)sqrt((double)p->spp);
    if (threads <= 0) threads = 1;
    if (threads == 1) worker(&J);
    else {
        pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
        for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, worker, &J);
        for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
        free(th);
    }
    if (rays_out) *rays_out = J.rays;
    return 0;
}

int port_trace_closest(void* sp, const float* rays, int64_t n, int depth, int max_depth, int32_t* prim, float* tout) {
    scene_t* s = (scene_t*)sp;
    if (!s || !rays) return 1;
    for (int64_t k = 0; k < n; ++k) {
        const float* R = rays + 8 * k;
        float t; int pi;
        int h = closest(s, V(R[0], R[1], R[2]), V(R[4], R[5], R[6]), R[3], R[7], depth == max_depth, 0, &t, &pi);
        if (prim) prim[k] = h ? s->prims[pi].gid : -1;
        if (tout) tout[k] = h ? t : INFINITY;
    }
    return 0;
}

int port_rng_draws(uint32_t seed, int64_t n, float* out) {
    rng_t r;
    minstd_seed(&r, seed);
    for (int64_t k = 0; k < n; ++k) out[k] = U(&r);
    return 0;
}

const char* port_last_error(void) { return g_err; }
