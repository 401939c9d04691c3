// rtc_trace.cuh - BVH traversal, primitive tests, materials, textures and the path loop.
//
// Every function states the reference function (flarive/CortexRaytracerCuda, core/src/...) whose
// arithmetic it reproduces.  The reference evaluates one virtual hit() per BVH node and primitive
// (bvh_node.cuh:110-118, hittable.cuh:47) with a ~120-byte hit_record copied per candidate; here the
// traversal is an iterative short-stack walk over a flattened SAH BVH2 whose inner loop computes only
// t, and the full hit record is computed once, for the winning primitive.
#pragma once

#include "rtc_dev.h"
#include "rtc_math.cuh"

namespace rtc {
inline namespace RTC_XP_NS {

// ------------------------------------------------------------------------------------------------
// random numbers
// ------------------------------------------------------------------------------------------------

// thrust::minstd_rand = linear_congruential_engine<uint32, 48271, 0, 2^31-1>
// (thrust/random/linear_congruential_engine.h) with uniform_real_distribution<float>(0, 1):
// U = float(x - 1) / (1.0f + float(2^31 - 3)) = float(x - 1) * 2^-31 (uniform_real_distribution.inl:61-74),
// which rounds to exactly 1.0f for the largest states.  The modular product uses 2^31 = 1 (mod m).
struct Minstd {
    uint32_t x;
    __device__ __forceinline__ void seed(uint32_t s) {
        uint32_t r = s % 2147483647u;
        x = r == 0u ? 1u : r;
    }
    __device__ __forceinline__ uint32_t next() {
        uint64_t p = (uint64_t)x * 48271ull;
        uint32_t r = (uint32_t)(p & 0x7fffffffull) + (uint32_t)(p >> 31);
        if (r >= 2147483647u) r -= 2147483647u;
        x = r;
        return r;
    }
    __device__ __forceinline__ float uniform() {
        return __uint2float_rn(next() - 1u) * 4.656612873077392578125e-10f;  // * 2^-31, exact
    }
};

// PCG32 (O'Neill 2014, "PCG: A Family of Simple Fast Space-Efficient Statistically Good Algorithms
// for Random Number Generation"): 64-bit LCG state, XSH-RR output.  Clean mode seeds one stream per
// (pixel, sample) from a hash of (seed, pixel, sample), so samples of a pixel are independent.
struct Pcg32 {
    uint64_t state, inc;
    __device__ __forceinline__ uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
    __device__ __forceinline__ float uniform() { return (float)(next() >> 8) * (1.0f / 16777216.0f); }
    __device__ __forceinline__ void seed(uint64_t initstate, uint64_t seq) {
        state = 0u;
        inc = (seq << 1u) | 1u;
        next();
        state += initstate;
        next();
    }
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {   // splitmix64 finaliser (Steele et al. 2014)
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// ------------------------------------------------------------------------------------------------
// scene loads: read-only, kept in L1 with the evict_last priority so that the path state the wavefront
// kernels stream (their slot records, loaded L2-only) does not push the BVH out of L1
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ float4 ld_scene(const float4* p) {
    float4 r;
    asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
        : "l"(p));
    return r;
}
__device__ __forceinline__ uint32_t ld_scene(const uint32_t* p) {
    uint32_t r;
    asm("ld.global.nc.L1::evict_last.u32 %0, [%1];" : "=r"(r) : "l"(p));
    return r;
}

// ------------------------------------------------------------------------------------------------
// hit record (the fields of hit_record the render path reads, misc/hit_record.cuh:8-38)
// ------------------------------------------------------------------------------------------------
struct Hit {
    float t;
    uint32_t item;     // leaf item (kind << 30 | index); 0xffffffff = none
    V3 p;              // hit_point
    V3 n;              // normal, facing the ray
    float u, v;
    bool front;
    bool sphere_uv;    // a sphere hit whose u, v are not computed yet (hit_uv computes them on first use)
    int mat;
};

// hit_record::set_face_normal (hit_record.cuh:34-38)
__device__ __forceinline__ void set_face_normal(Hit& h, V3 dir, V3 outward) {
    h.front = dot(dir, outward) < 0.0f;
    h.n = h.front ? outward : neg(outward);
}

// ------------------------------------------------------------------------------------------------
// primitive t tests: same arithmetic and interval rule as the reference's hit()
// ------------------------------------------------------------------------------------------------

// sphere::hit (sphere.cuh:111-135): half-b quadratic, strict interval (interval::surrounds).
__device__ __forceinline__ bool sphere_t(float4 s, V3 o, V3 d, float tmin, float tmax, float& t) {
    V3 c = v3(s.x, s.y, s.z);
    V3 oc = sub(o, c);
    float a = lensq(d);
    float half_b = oc.x * d.x + oc.y * d.y + oc.z * d.z;   // dot_vector (vector3.cuh:92-94)
    float cc = lensq(oc) - s.w * s.w;
    float disc = half_b * half_b - a * cc;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float root = (-half_b - sq) / a;
    if (!(tmin < root && root < tmax)) {
        root = (-half_b + sq) / a;
        if (!(tmin < root && root < tmax)) return false;
    }
    t = root;
    return true;
}

// Clean mode's sphere test: the same quadratic in double.  In float, |o-c|^2 - r^2 cancels
// catastrophically for large spheres (a ground sphere of radius 1000: ulp(1e6) = 0.06), so hit
// distances are off by ~3e-5, more than tmin and the robust offset, and bounce rays re-hit their own
// surface: the float image is ~5% darker than the double-precision estimate on such scenes.  The
// reference has the same defect, which compat mode keeps.
__device__ __forceinline__ bool sphere_t_exact(float4 s, V3 o, V3 d, float tmin, float tmax, float& t) {
    const double ox = (double)o.x - (double)s.x, oy = (double)o.y - (double)s.y, oz = (double)o.z - (double)s.z;
    const double dx = d.x, dy = d.y, dz = d.z;
    const double a = dx * dx + dy * dy + dz * dz;
    const double hb = ox * dx + oy * dy + oz * dz;
    const double cc = ox * ox + oy * oy + oz * oz - (double)s.w * (double)s.w;
    const double disc = hb * hb - a * cc;
    if (disc < 0.0) return false;
    const double sq = sqrt(disc);
    double root = (-hb - sq) / a;
    if (!((double)tmin < root && root < (double)tmax)) {
        root = (-hb + sq) / a;
        if (!((double)tmin < root && root < (double)tmax)) return false;
    }
    t = (float)root;
    return true;
}

// quad::hit (quad.cuh:100-133) and directional_light::hit (directional_light.cuh:76-120).
// q0 = (n, D), q1 = (Q or P), q2 = u, q3 = v, q4 = w.  centred: light interior test on [-0.5, 0.5].
__device__ __forceinline__ bool planar_t(float4 q0, float4 q1, float4 q2, float4 q3, float4 q4, V3 o, V3 d,
                                         float tmin, float tmax, bool centred, float& t, float& alpha,
                                         float& beta) {
    V3 n = v3(q0.x, q0.y, q0.z);
    float denom = dot(n, d);
    if ((double)fabsf(denom) < 1e-8) return false;          // fabs(denom) < 1e-8 (double literal)
    float tt = (q0.w - dot(n, o)) / denom;
    if (!(tmin <= tt && tt <= tmax)) return false;          // interval::contains
    V3 ip = at(o, d, tt);
    V3 pl = sub(ip, v3(q1.x, q1.y, q1.z));
    V3 w = v3(q4.x, q4.y, q4.z);
    float a = dot(w, cross(pl, v3(q3.x, q3.y, q3.z)));
    float b = dot(w, cross(v3(q2.x, q2.y, q2.z), pl));
    if (centred) {
        if ((a < -0.5f) || (0.5f < a) || (b < -0.5f) || (0.5f < b)) return false;
    } else {
        if ((a < 0.0f) || (1.0f < a) || (b < 0.0f) || (1.0f < b)) return false;
    }
    t = tt;
    alpha = a;
    beta = b;
    return true;
}

// triangle::hit (triangle.cuh:130-160): Moller-Trumbore, |det| < 1e-6 rejected, inclusive bounds.
__device__ __forceinline__ bool tri_t(float4 a0, float4 a1, float4 a2, V3 o, V3 d, float tmin, float tmax,
                                      float& t, float& bu, float& bv) {
    V3 v0 = v3(a0.x, a0.y, a0.z), e1 = v3(a1.x, a1.y, a1.z), e2 = v3(a2.x, a2.y, a2.z);
    V3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (fabsf(det) < 0.000001f) return false;
    float inv_det = 1.0f / det;
    V3 tv = sub(o, v0);
    float u = dot(tv, pv) * inv_det;
    if (u < 0.0f || u > 1.0f) return false;
    V3 qv = cross(tv, e1);
    float v = dot(d, qv) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    float tt = dot(e2, qv) * inv_det;
    if (tt < tmin || tt > tmax) return false;
    t = tt;
    bu = u;
    bv = v;
    return true;
}

// ------------------------------------------------------------------------------------------------
// BVH traversal (closest hit)
// ------------------------------------------------------------------------------------------------
struct TraceStats {
    uint32_t nodes, prims;
};

// Packed pairs of floats for the box tests (sm_100's f32x2 arithmetic: one instruction, two lanes, each
// rounded as the scalar instruction rounds it) and three-input min / max (sm_100).  RTC_WIDE_PACKED=0 /
// RTC_BINARY_PACKED=0 build the scalar form of the same arithmetic for the 8-wide / binary nodes.
#ifndef RTC_WIDE_PACKED
#define RTC_WIDE_PACKED 1
#endif
#ifndef RTC_BINARY_PACKED
#define RTC_BINARY_PACKED 1
#endif
typedef unsigned long long F2;
__device__ __forceinline__ F2 f2(float lo, float hi) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void split_f2(F2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ F2 fma_f2(F2 a, F2 b, F2 c) {
    F2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
// bytes c and c + 1 (c = 0 or 2) of `w` as a pair of floats, as byte_f does for one
__device__ __forceinline__ F2 bytes_f2(uint32_t w, int c) {
    const F2 two23 = 0x4B0000004B000000ull;
    const F2 v = f2(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7650u | (uint32_t)c)),
                    __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7650u | (uint32_t)(c + 1))));
    F2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(v), "l"(two23));
    return d;
}
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

__device__ __forceinline__ bool slab2(const float4 n0, const float4 n1, const float4 n2, V3 inv, V3 oi,
                                      float tmin, float tmax, float& tl, float& tr, bool& hr) {
    // t = lo*inv - o*inv, one FMA per bound; boxes are padded on the host so rounding never culls.
#if RTC_BINARY_PACKED
    // each float4 holds a child's (lo, hi) pairs, so one f32x2 FMA gives both planes of an axis
    const F2 ix = f2(inv.x, inv.x), iy = f2(inv.y, inv.y), iz = f2(inv.z, inv.z);
    const F2 ox = f2(-oi.x, -oi.x), oy = f2(-oi.y, -oi.y), oz = f2(-oi.z, -oi.z);
    float l0x, l1x, l0y, l1y, l0z, l1z, r0x, r1x, r0y, r1y, r0z, r1z;
    split_f2(fma_f2(f2(n0.x, n0.y), ix, ox), l0x, l1x);
    split_f2(fma_f2(f2(n0.z, n0.w), iy, oy), l0y, l1y);
    split_f2(fma_f2(f2(n2.x, n2.y), iz, oz), l0z, l1z);
    split_f2(fma_f2(f2(n1.x, n1.y), ix, ox), r0x, r1x);
    split_f2(fma_f2(f2(n1.z, n1.w), iy, oy), r0y, r1y);
    split_f2(fma_f2(f2(n2.z, n2.w), iz, oz), r0z, r1z);
    const float lin = fmax3(fminf(l0x, l1x), fminf(l0y, l1y), fmaxf(fminf(l0z, l1z), tmin));
    const float lout = fmin3(fmaxf(l0x, l1x), fmaxf(l0y, l1y), fminf(fmaxf(l0z, l1z), tmax));
    const float rin = fmax3(fminf(r0x, r1x), fminf(r0y, r1y), fmaxf(fminf(r0z, r1z), tmin));
    const float rout = fmin3(fmaxf(r0x, r1x), fmaxf(r0y, r1y), fminf(fmaxf(r0z, r1z), tmax));
#else
    float l0x = __fmaf_rn(n0.x, inv.x, -oi.x), l1x = __fmaf_rn(n0.y, inv.x, -oi.x);
    float l0y = __fmaf_rn(n0.z, inv.y, -oi.y), l1y = __fmaf_rn(n0.w, inv.y, -oi.y);
    float l0z = __fmaf_rn(n2.x, inv.z, -oi.z), l1z = __fmaf_rn(n2.y, inv.z, -oi.z);
    float r0x = __fmaf_rn(n1.x, inv.x, -oi.x), r1x = __fmaf_rn(n1.y, inv.x, -oi.x);
    float r0y = __fmaf_rn(n1.z, inv.y, -oi.y), r1y = __fmaf_rn(n1.w, inv.y, -oi.y);
    float r0z = __fmaf_rn(n2.z, inv.z, -oi.z), r1z = __fmaf_rn(n2.w, inv.z, -oi.z);
    float lin = fmaxf(fmaxf(fminf(l0x, l1x), fminf(l0y, l1y)), fmaxf(fminf(l0z, l1z), tmin));
    float lout = fminf(fminf(fmaxf(l0x, l1x), fmaxf(l0y, l1y)), fminf(fmaxf(l0z, l1z), tmax));
    float rin = fmaxf(fmaxf(fminf(r0x, r1x), fminf(r0y, r1y)), fmaxf(fminf(r0z, r1z), tmin));
    float rout = fminf(fminf(fmaxf(r0x, r1x), fmaxf(r0y, r1y)), fminf(fmaxf(r0z, r1z), tmax));
#endif
    tl = lin;
    tr = rin;
    hr = rin <= rout;
    return lin <= lout;
}

// ------------------------------------------------------------------------------------------------
// transformed primitives and box faces
// ------------------------------------------------------------------------------------------------
// glm mat4 * vec4 (glm/detail/type_mat4x4.inl:560-571) for a rotation matrix, whose fourth column is
// (0, 0, 0, 1): component i = (m0_i x + m1_i y) + (m2_i z + m3_i w), and m3_i w is +0 for i < 3.
__device__ __forceinline__ V3 rot_apply(float4 m0, float4 m1, float4 m2, V3 v) {
    return v3((m0.x * v.x + m1.x * v.y) + (m2.x * v.z + 0.0f), (m0.y * v.x + m1.y * v.y) + (m2.y * v.z + 0.0f),
              (m0.z * v.x + m1.z * v.y) + (m2.z * v.z + 0.0f));
}

// World ray -> object space through scale, rotate, translate (scale.cuh, rotate.cuh, translate.cuh hit()).
__device__ __forceinline__ void xf_to_object(const DevScene& S, int32_t xi, V3& o, V3& d) {
    const float4* x = S.xf + 8 * (size_t)xi;
    const float4 h0 = __ldg(x);
    const uint32_t fl = __float_as_uint(h0.w);
    if (fl & 4u) {
        const float4 sc = __ldg(x + 1);
        o = v3(o.x / sc.x, o.y / sc.y, o.z / sc.z);
        d = v3(d.x / sc.x, d.y / sc.y, d.z / sc.z);
    }
    if (fl & 2u) {
        const float4 m0 = __ldg(x + 2), m1 = __ldg(x + 3), m2 = __ldg(x + 4);
        o = rot_apply(m0, m1, m2, o);
        d = rot_apply(m0, m1, m2, d);
    }
    if (fl & 1u) o = v3(o.x - h0.x, o.y - h0.y, o.z - h0.z);
}

// Hit point and normal back to world space: translate (+t), rotate (forward matrix), scale (p * s,
// normal unit_vector(n / s)).
__device__ __forceinline__ void xf_to_world(const DevScene& S, int32_t xi, V3& p, V3& n) {
    const float4* x = S.xf + 8 * (size_t)xi;
    const float4 h0 = __ldg(x);
    const uint32_t fl = __float_as_uint(h0.w);
    if (fl & 1u) p = v3(p.x + h0.x, p.y + h0.y, p.z + h0.z);
    if (fl & 2u) {
        const float4 m0 = __ldg(x + 5), m1 = __ldg(x + 6), m2 = __ldg(x + 7);
        p = rot_apply(m0, m1, m2, p);
        n = rot_apply(m0, m1, m2, n);
    }
    if (fl & 4u) {
        const float4 sc = __ldg(x + 1);
        p = v3(p.x * sc.x, p.y * sc.y, p.z * sc.z);
        n = unit(v3(n.x / sc.x, n.y / sc.y, n.z / sc.z));
    }
}

// xy_rect / xz_rect / yz_rect::hit (aarect.cuh): t = (k - o_a) / d_a in [tmin, tmax] inclusive, then the
// two in-plane coordinates inside the rectangle, bounds inclusive.
__device__ __forceinline__ bool rect_t(float4 r0, float4 r1, V3 o, V3 d, float tmin, float tmax, float& t, float& a,
                                       float& b) {
    const int axis = __float_as_int(r1.y);
    const float oa = axis == 0 ? o.z : axis == 1 ? o.y : o.x;
    const float da = axis == 0 ? d.z : axis == 1 ? d.y : d.x;
    t = (r1.x - oa) / da;
    if (t < tmin || t > tmax) return false;
    const float o0 = axis == 2 ? o.y : o.x, d0 = axis == 2 ? d.y : d.x;
    const float o1 = axis == 0 ? o.y : o.z, d1 = axis == 0 ? d.y : d.z;
    a = o0 + t * d0;
    b = o1 + t * d1;
    return !(a < r0.x || a > r0.y || b < r0.z || b > r0.w);
}

// Tests every item of one leaf against [tmin, best_t].  EXACT: clean mode's double-precision sphere test.
// A leaf of the xprim BVH: transformed primitives and box faces, each tested on its object-space ray.
template <bool EXACT>
__device__ __forceinline__ void test_leaf_xprims(const DevScene& S, int32_t child, V3 o, V3 d, float tmin,
                                                 float& best_t, uint32_t& best_item, TraceStats& st,
                                                 uint32_t& status) {
    const uint32_t enc = (uint32_t)(~child);
    const uint32_t first = enc >> LEAF_COUNT_BITS, cnt = enc & MAX_LEAF;
    if (first + cnt > S.num_xitems) { status |= STATUS_BAD_ITEM; return; }
    for (uint32_t k = 0; k < cnt; ++k) {
        const uint32_t it = ld_scene(S.xitems + first + k);
        const uint32_t idx = it & ITEM_INDEX_MASK;
        st.prims++;
        if ((it >> ITEM_KIND_SHIFT) != ITEM_XPRIM || idx >= S.num_xprim) { status |= STATUS_BAD_ITEM; continue; }
        const int4 x = __ldg(S.xprim + idx);
        V3 ro = o, rd = d;
        if (x.x >= 0) {
            if ((uint32_t)x.x >= S.num_xf) { status |= STATUS_BAD_ITEM; continue; }
            xf_to_object(S, x.x, ro, rd);
        }
        const uint32_t in = (uint32_t)x.z;
        float t;
        bool h = false;
        switch (x.y) {
        case ITEM_SPHERE: {
            if (in >= S.num_sph) { status |= STATUS_BAD_ITEM; break; }
            const float4 sp = ld_scene(S.sph + in);
            h = EXACT ? sphere_t_exact(sp, ro, rd, tmin, best_t, t) : sphere_t(sp, ro, rd, tmin, best_t, t);
        } break;
        case ITEM_QUAD: {
            if (in >= S.num_quad) { status |= STATUS_BAD_ITEM; break; }
            const float4* q = S.quad + 5 * (size_t)in;
            float a, b;
            h = planar_t(__ldg(q), __ldg(q + 1), __ldg(q + 2), __ldg(q + 3), __ldg(q + 4), ro, rd, tmin, best_t, false, t, a, b);
        } break;
        case ITEM_TRI: {
            if (in >= S.num_tri) { status |= STATUS_BAD_ITEM; break; }
            const float4* p = S.tri + 3 * (size_t)in;
            float bu, bv;
            h = tri_t(ld_scene(p), ld_scene(p + 1), ld_scene(p + 2), ro, rd, tmin, best_t, t, bu, bv);
        } break;
        case XPRIM_RECT: {
            if (in >= S.num_rect) { status |= STATUS_BAD_ITEM; break; }
            float a, b;
            h = rect_t(__ldg(S.rect + 2 * (size_t)in), __ldg(S.rect + 2 * (size_t)in + 1), ro, rd, tmin, best_t, t, a, b);
        } break;
        default: status |= STATUS_BAD_ITEM; break;
        }
        if (h) {
            best_t = t;
            best_item = it;
        }
    }
}

// Items [first, first + cnt) of an item list (`items`, or `items8` for the 8-wide nodes; both hold
// num_items entries) against [tmin, best_t].
template <bool EXACT>
__device__ __forceinline__ void test_items(const DevScene& S, const uint32_t* items, uint32_t first, uint32_t cnt,
                                           V3 o, V3 d, float tmin, float& best_t, uint32_t& best_item,
                                           bool hide_invisible, TraceStats& st, uint32_t& status) {
    if (first + cnt > S.num_items) { status |= STATUS_BAD_ITEM; return; }
    for (uint32_t k = 0; k < cnt; ++k) {
        uint32_t it = ld_scene(items + first + k);
        uint32_t kind = it >> ITEM_KIND_SHIFT, idx = it & ITEM_INDEX_MASK;
        float t;
        st.prims++;
        switch (kind) {
        case ITEM_TRI: {
            if (idx >= S.num_tri) { status |= STATUS_BAD_ITEM; break; }
            const float4* p = S.tri + 3 * (size_t)idx;
            float bu, bv;
            if (tri_t(ld_scene(p), ld_scene(p + 1), ld_scene(p + 2), o, d, tmin, best_t, t, bu, bv)) { best_t = t; best_item = it; }
        } break;
        case ITEM_SPHERE: {
            if (idx >= S.num_sph) { status |= STATUS_BAD_ITEM; break; }
            const float4 sp = ld_scene(S.sph + idx);
            if (EXACT ? sphere_t_exact(sp, o, d, tmin, best_t, t) : sphere_t(sp, o, d, tmin, best_t, t)) {
                best_t = t;
                best_item = it;
            }
        } break;
        case ITEM_QUAD: {
            if (idx >= S.num_quad) { status |= STATUS_BAD_ITEM; break; }
            const float4* q = S.quad + 5 * (size_t)idx;
            float a, b;
            if (planar_t(__ldg(q), __ldg(q + 1), __ldg(q + 2), __ldg(q + 3), __ldg(q + 4), o, d, tmin, best_t, false, t, a, b)) {
                best_t = t;
                best_item = it;
            }
        } break;
        case ITEM_LIGHT: {
            if (idx >= S.num_lights) { status |= STATUS_BAD_ITEM; break; }
            const float4* q = S.light + 6 * (size_t)idx;
            float a, b;
            const float4 q3 = __ldg(q + 3), q4 = __ldg(q + 4);
            bool hitl;
            if (q4.w < 0.0f) {
                // omni_light::hit / spot_light::hit (omni_light.cuh:55-83): the sphere quadratic, strict
                const float4 sp = __ldg(q);
                hitl = EXACT ? sphere_t_exact(sp, o, d, tmin, best_t, t) : sphere_t(sp, o, d, tmin, best_t, t);
            } else {
                hitl = planar_t(__ldg(q), __ldg(q + 1), __ldg(q + 2), q3, q4, o, d, tmin, best_t, true, t, a, b);
            }
            // "Hide light source": invisible lights are skipped when depth == max_depth
            // (directional_light.cuh:106, omni_light.cuh:76-80)
            if (hitl && !(q3.w != 0.0f && hide_invisible)) { best_t = t; best_item = it; }
        } break;
        default: status |= STATUS_BAD_ITEM; break;
        }
    }
}

// A binary leaf: child = ~((first << LEAF_COUNT_BITS) | count) over `items`.
template <bool EXACT>
__device__ __forceinline__ void test_leaf(const DevScene& S, int32_t child, V3 o, V3 d, float tmin, float& best_t,
                                          uint32_t& best_item, bool hide_invisible, TraceStats& st,
                                          uint32_t& status) {
    const uint32_t enc = (uint32_t)(~child);
    test_items<EXACT>(S, S.items, enc >> LEAF_COUNT_BITS, enc & MAX_LEAF, o, d, tmin, best_t, best_item,
                      hide_invisible, st, status);
}

// Direction component for the slab tests' reciprocal.  The slab distance is fma(lo, 1/d, -o/d); with a
// zero component the two infinite products cancel to NaN or collapse to -inf by the SIGNS of lo and o,
// not by whether o lies between the slab's planes, so a box whose slab holds the origin could be culled
// (the reference subtracts first, (lo - o) / d, and keeps it).  Components below 1e-20 in magnitude are
// traced as +-1e-20: the reciprocal stays finite, a slab that holds the origin spans about
// [-1e20 |lo - o|, +1e20 |hi - o|], and one that does not lies beyond any finite hit.  Other components
// are unchanged, so every other ray walks the tree exactly as before.
__device__ __forceinline__ float slab_dir(float x) { return fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x; }

// Byte `c` (0-3) of `w` as a float: the byte becomes the low mantissa byte of 2^23, and subtracting
// 2^23 leaves exactly its value (two full-rate instructions instead of an integer-to-float conversion).
__device__ __forceinline__ float byte_f(uint32_t w, int c) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7650u | (uint32_t)c)) - 8388608.0f;
}

// An 8-wide node's link word (child base, item base, link bytes 0-3, link bytes 4-7).
__device__ __forceinline__ int4 ld_links(const float4* p) {
    const float4 v = ld_scene(p);
    return make_int4(__float_as_int(v.x), __float_as_int(v.y), __float_as_int(v.z), __float_as_int(v.w));
}

// Bits of an 8-bit mask moved from position s to position s ^ oct.
__device__ __forceinline__ uint32_t octant_order(uint32_t h, uint32_t oct) {
    if (oct & 1u) h = ((h & 0x55u) << 1) | ((h >> 1) & 0x55u);
    if (oct & 2u) h = ((h & 0x33u) << 2) | ((h >> 2) & 0x33u);
    if (oct & 4u) h = ((h & 0x0fu) << 4) | ((h >> 4) & 0x0fu);
    return h;
}

// Closest hit through the 8-wide nodes (compressed wide layout, after Ylitie, Karras and Laine, HPG
// 2017).  A visit loads one 80-byte node and tests its children's quantised boxes: on each axis the
// bound p + q * 2^e gives the distance fma(q, 2^e / d, (p - o) / d), the same rounding model as the
// binary slab (the step is a power of two, so 2^e / d is exact).  The ray's direction signs pick, per
// axis, which of a child's two bounds is its entry and which its exit plane, so a child costs six
// distances and no min/max per axis.  The hit children form a group: (node, mask of hit slots), the
// mask in visiting order (bit j = slot j ^ oct, near corner first).  The walk takes the group's next
// child: a leaf is tested in place; for an inner child the rest of the group is pushed as one 32-bit
// entry (node << 8 | mask) and the child's own group replaces it.  No sort, no distances on the stack:
// at most one entry per level.
template <bool EXACT>
__device__ __forceinline__ bool closest_hit8(const DevScene& S, V3 o, V3 d, V3 inv, V3 oi, float tmin, float tmax,
                                             bool hide_invisible, float& t_out, uint32_t& item_out,
                                             TraceStats& st, uint32_t& status) {
    float best_t = tmax;
    uint32_t best_item = 0xffffffffu;
    // direction sign bits; slab_dir keeps the sign of a zero component, so inv has it too
    const uint32_t oct = (inv.x < 0.0f ? 1u : 0u) | (inv.y < 0.0f ? 2u : 0u) | (inv.z < 0.0f ? 4u : 0u);
    uint32_t stk[TRAVERSAL_STACK8];
    int sp = 0;
    uint32_t node = 0;       // the current group: its node, the slots still to take (visiting order)
    uint32_t hits = 0;       // and the node's links (child base, item base, link bytes)
    int4 links = make_int4(0, 0, 0, 0);
    int32_t visit = 0;       // node to visit at the top of the next pass, -1: none
    // A walk visits each node and leaf at most once; more visits than that mean malformed links, and
    // the walk stops with STATUS_TIMEOUT instead of running on.
    const uint32_t visit_limit = 2u * (S.num_nodes8 + S.num_items) + 64u;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > visit_limit) { status |= STATUS_TIMEOUT; break; }
        if (visit >= 0) {
            if ((uint32_t)visit >= S.num_nodes8) { status |= STATUS_BAD_ITEM; break; }
            node = (uint32_t)visit;
            visit = -1;
            const float4* np = S.nodes8 + 5 * (size_t)node;
            const float4 h = ld_scene(np), qx = ld_scene(np + 2), qy = ld_scene(np + 3), qz = ld_scene(np + 4);
            links = ld_links(np + 1);
            st.nodes++;
            const uint32_t hdr = __float_as_uint(h.w);
            const float ax = __uint_as_float((hdr & 0xffu) << 23) * inv.x;
            const float ay = __uint_as_float(((hdr >> 8) & 0xffu) << 23) * inv.y;
            const float az = __uint_as_float(((hdr >> 16) & 0xffu) << 23) * inv.z;
            const float bx = __fmaf_rn(h.x, inv.x, -oi.x), by = __fmaf_rn(h.y, inv.y, -oi.y),
                        bz = __fmaf_rn(h.z, inv.z, -oi.z);
            // entry (n) and exit (f) bound words per axis: the low bounds are the entry planes where the
            // direction is positive, the high bounds where it is negative
            const uint32_t nx0 = __float_as_uint((oct & 1u) ? qx.z : qx.x), nx1 = __float_as_uint((oct & 1u) ? qx.w : qx.y);
            const uint32_t fx0 = __float_as_uint((oct & 1u) ? qx.x : qx.z), fx1 = __float_as_uint((oct & 1u) ? qx.y : qx.w);
            const uint32_t ny0 = __float_as_uint((oct & 2u) ? qy.z : qy.x), ny1 = __float_as_uint((oct & 2u) ? qy.w : qy.y);
            const uint32_t fy0 = __float_as_uint((oct & 2u) ? qy.x : qy.z), fy1 = __float_as_uint((oct & 2u) ? qy.y : qy.w);
            const uint32_t nz0 = __float_as_uint((oct & 4u) ? qz.z : qz.x), nz1 = __float_as_uint((oct & 4u) ? qz.w : qz.y);
            const uint32_t fz0 = __float_as_uint((oct & 4u) ? qz.x : qz.z), fz1 = __float_as_uint((oct & 4u) ? qz.y : qz.w);
            uint32_t hs = 0;
#if RTC_WIDE_PACKED
            // two children per instruction: packed f32x2 subtract and FMA, the same roundings per lane
            const F2 ax2 = f2(ax, ax), ay2 = f2(ay, ay), az2 = f2(az, az);
            const F2 bx2 = f2(bx, bx), by2 = f2(by, by), bz2 = f2(bz, bz);
#pragma unroll
            for (int c = 0; c < 8; c += 2) {
                const int b = c & 3;
                const F2 tnx = fma_f2(bytes_f2(c < 4 ? nx0 : nx1, b), ax2, bx2);
                const F2 tfx = fma_f2(bytes_f2(c < 4 ? fx0 : fx1, b), ax2, bx2);
                const F2 tny = fma_f2(bytes_f2(c < 4 ? ny0 : ny1, b), ay2, by2);
                const F2 tfy = fma_f2(bytes_f2(c < 4 ? fy0 : fy1, b), ay2, by2);
                const F2 tnz = fma_f2(bytes_f2(c < 4 ? nz0 : nz1, b), az2, bz2);
                const F2 tfz = fma_f2(bytes_f2(c < 4 ? fz0 : fz1, b), az2, bz2);
                float nx[2], ny[2], nz[2], fx[2], fy[2], fz[2];
                split_f2(tnx, nx[0], nx[1]);
                split_f2(tny, ny[0], ny[1]);
                split_f2(tnz, nz[0], nz[1]);
                split_f2(tfx, fx[0], fx[1]);
                split_f2(tfy, fy[0], fy[1]);
                split_f2(tfz, fz[0], fz[1]);
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const float tn = fmax3(nx[k], ny[k], fmaxf(nz[k], tmin));
                    const float tf = fmin3(fx[k], fy[k], fminf(fz[k], best_t));
                    hs |= (tn <= tf ? 1u : 0u) << (c + k);
                }
            }
#else
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int b = c & 3;
                const float tnx = __fmaf_rn(byte_f(c < 4 ? nx0 : nx1, b), ax, bx);
                const float tfx = __fmaf_rn(byte_f(c < 4 ? fx0 : fx1, b), ax, bx);
                const float tny = __fmaf_rn(byte_f(c < 4 ? ny0 : ny1, b), ay, by);
                const float tfy = __fmaf_rn(byte_f(c < 4 ? fy0 : fy1, b), ay, by);
                const float tnz = __fmaf_rn(byte_f(c < 4 ? nz0 : nz1, b), az, bz);
                const float tfz = __fmaf_rn(byte_f(c < 4 ? fz0 : fz1, b), az, bz);
                const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
                const float tf = fminf(fminf(tfx, tfy), fminf(tfz, best_t));
                hs |= (tn <= tf ? 1u : 0u) << c;
            }
#endif
            hits = octant_order(hs & (hdr >> 24), oct);
        }
        if (hits == 0u) {
            if (sp == 0) break;
            const uint32_t e = stk[--sp];
            node = e >> 8;
            hits = e & 0xffu;
            links = ld_links(S.nodes8 + 5 * (size_t)node + 1);
        }
        // the group's next child
        const uint32_t slot = (uint32_t)(__ffs(hits) - 1) ^ oct;
        hits &= hits - 1u;
        const uint32_t lb = ((uint32_t)(slot < 4u ? links.z : links.w) >> (8u * (slot & 3u))) & 0xffu;
        if (lb & 0x80u) {
            if (hits) {
                if (sp >= TRAVERSAL_STACK8) { status |= STATUS_STACK_OVERFLOW; break; }
                stk[sp++] = (node << 8) | hits;
            }
            visit = links.x + (int32_t)(lb & 7u);
        } else {
            test_items<EXACT>(S, S.items8, (uint32_t)links.y + (lb & 31u), ((lb >> 5) & 3u) + 1u, o, d, tmin, best_t,
                              best_item, hide_invisible, st, status);
        }
    }
    t_out = best_t;
    item_out = best_item;
    return best_item != 0xffffffffu;
}

// The xprim BVH (binary, `xnodes` / `xitems`) against [tmin, best_t]: updates best_t / best_item and
// returns whether any hit is held.  Same node layout and walk as the binary traversal below.
template <bool EXACT>
__device__ __forceinline__ bool closest_hit_xprims(const DevScene& S, V3 o, V3 d, V3 inv, V3 oi, float tmin,
                                                float& best_t, uint32_t& best_item, TraceStats& st,
                                                uint32_t& status) {
    int32_t stack[TRAVERSAL_STACK];
    int sp = 0;
    int32_t node = 0;
    for (;;) {
        const float4* np = S.xnodes + 4 * (size_t)node;
        float4 n0 = ld_scene(np), n1 = ld_scene(np + 1), n2 = ld_scene(np + 2), n3 = ld_scene(np + 3);
        st.nodes++;
        int32_t cl = __float_as_int(n3.x), cr = __float_as_int(n3.y);
        float tl, tr;
        bool hr;
        bool hl = slab2(n0, n1, n2, inv, oi, tmin, best_t, tl, tr, hr);
        if (hl && cl < 0) { test_leaf_xprims<EXACT>(S, cl, o, d, tmin, best_t, best_item, st, status); hl = false; }
        if (hr && cr < 0) { test_leaf_xprims<EXACT>(S, cr, o, d, tmin, best_t, best_item, st, status); hr = false; }
        if (hl && hr) {
            int32_t nearc = tl <= tr ? cl : cr;
            int32_t farc = tl <= tr ? cr : cl;
            if (sp >= TRAVERSAL_STACK) { status |= STATUS_STACK_OVERFLOW; break; }
            stack[sp++] = farc;
            node = nearc;
        } else if (hl) {
            node = cl;
        } else if (hr) {
            node = cr;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
        if ((uint32_t)node >= S.num_xnodes) { status |= STATUS_BAD_ITEM; break; }
    }
    return best_item != 0xffffffffu;
}

// Closest hit in [tmin, tmax] over the whole scene (the reference's world.hit through the BVH).
// EXACT: clean mode (double-precision sphere test).  WIDE: walk the 8-wide nodes when the scene
// carries them (only the extend kernel is built with it, so the other kernels carry no code for it).
template <bool EXACT = false, bool WIDE = false>
__device__ __forceinline__ bool closest_hit(const DevScene& S, V3 o, V3 d, float tmin, float tmax,
                                            bool hide_invisible, float& t_out, uint32_t& item_out,
                                            TraceStats& st, uint32_t& status) {
    // A zero direction meets no primitive: every test of the reference's hit() rejects it (0/0 roots,
    // zero denominator, zero determinant), so it misses without a walk.  Such rays are common: a
    // lambertian bounce with an empty light list scatters along a zero vector.
    if (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) {
        t_out = tmax;
        item_out = 0xffffffffu;
        return false;
    }
    V3 inv = v3(1.0f / slab_dir(d.x), 1.0f / slab_dir(d.y), 1.0f / slab_dir(d.z));
    if constexpr (WIDE) {
        if (S.nodes8) {
            V3 oi8 = v3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
            bool h = closest_hit8<EXACT>(S, o, d, inv, oi8, tmin, tmax, hide_invisible, t_out, item_out, st, status);
#if RTC_XP
            if (S.num_xnodes) h = closest_hit_xprims<EXACT>(S, o, d, inv, oi8, tmin, t_out, item_out, st, status);
#endif
            return h;
        }
    }
    V3 oi = v3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
    float best_t = tmax;
    uint32_t best_item = 0xffffffffu;
    int32_t stack[TRAVERSAL_STACK];
    int sp = 0;
    int32_t node = 0;
    for (;;) {
#if RTC_XP
        if (S.num_nodes == 0) break;   // every primitive is transformed (xprim BVH only)
#endif
        const float4* np = S.nodes + 4 * (size_t)node;
        float4 n0 = ld_scene(np), n1 = ld_scene(np + 1), n2 = ld_scene(np + 2), n3 = ld_scene(np + 3);
        st.nodes++;
        int32_t cl = __float_as_int(n3.x), cr = __float_as_int(n3.y);
        float tl, tr;
        bool hr;
        bool hl = slab2(n0, n1, n2, inv, oi, tmin, best_t, tl, tr, hr);
        if (hl && cl < 0) { test_leaf<EXACT>(S, cl, o, d, tmin, best_t, best_item, hide_invisible, st, status); hl = false; }
        if (hr && cr < 0) { test_leaf<EXACT>(S, cr, o, d, tmin, best_t, best_item, hide_invisible, st, status); hr = false; }
        if (hl && hr) {
            int32_t nearc = tl <= tr ? cl : cr;
            int32_t farc = tl <= tr ? cr : cl;
            if (sp >= TRAVERSAL_STACK) { status |= STATUS_STACK_OVERFLOW; break; }
            stack[sp++] = farc;
            node = nearc;
        } else if (hl) {
            node = cl;
        } else if (hr) {
            node = cr;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
        if ((uint32_t)node >= S.num_nodes) { status |= STATUS_BAD_ITEM; break; }
    }
    t_out = best_t;
    item_out = best_item;
    // transformed primitives and box faces live in their own BVH, walked after the first one against the
    // best hit so far; scenes without them skip it (and their traversal loop carries none of its registers)
#if RTC_XP
    if (S.num_xnodes) return closest_hit_xprims<EXACT>(S, o, d, inv, oi, tmin, t_out, item_out, st, status);
#endif
    return best_item != 0xffffffffu;
}

// Full hit record of the winning item: the part of each reference hit() that runs after the
// interval test (sphere.cuh:137-165, quad.cuh:122-132, directional_light.cuh:113-120,
// triangle.cuh:160-184).
// fmod(x, 1) (the wraps of uvmapping.cuh): x - trunc(x) carries the sign of x and is exact - the
// fractional part of a float is representable, and |x| >= 2^23 is an integer - so this equals fmodf(x,
// 1.0f) for every x (NaN for infinities and NaN, zero of x's sign for integers) in three instructions
// where fmodf's general algorithm inlines a loop into every kernel that finalises a hit.
__device__ __forceinline__ float fmod1(float x) { return copysignf(x - truncf(x), x); }

// get_triangle_uv (uvmapping.cuh:415-429) at a triangle hit's point: get_barycenter's barycentrics
// (math_utils.cuh:73-86) over v0, v1 = v0 + e1, v2 = v0 + e2, then calculateTextureCoordinate
// (uvmapping.cuh:435-447) with its wrap into [0, 1).  The reference passes the hit record's previous
// hit point (triangle.cuh:162), which depends on the BVH's visit order; this uses the hit's own.
__device__ __forceinline__ void tri_uv_at(const DevScene& S, uint32_t idx, float4 a0, float4 a1, float4 a2, Hit& h) {
    const V3 e1 = v3(a1.x, a1.y, a1.z), e2 = v3(a2.x, a2.y, a2.z), p2 = sub(h.p, v3(a0.x, a0.y, a0.z));
    const float d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(p2, e1), d21 = dot(p2, e2);
    const float denom = d00 * d11 - d01 * d01;
    const float bv = (d11 * d20 - d01 * d21) / denom;
    const float bw = (d00 * d21 - d01 * d20) / denom;
    const float bu = 1.0f - bv - bw;
    const float4 t0 = __ldg(S.tri_uv + 2 * (size_t)idx), t1 = __ldg(S.tri_uv + 2 * (size_t)idx + 1);
    float tu = bu * t0.x + bv * t0.z + (1.0f - bu - bv) * t1.x;
    float tv = bu * t0.y + bv * t0.w + (1.0f - bu - bv) * t1.y;
    tu = fmod1(tu);
    tv = fmod1(tv);
    if (tu < 0.0f) tu += 1.0f;
    if (tv < 0.0f) tv += 1.0f;
    h.u = tu;
    h.v = tv;
}

// get_sphere_uv (uvmapping.cuh:204-228) with the default mapping (repeat 1, scale 1, offset 0) of a
// sphere hit's outward normal, computed the first time a texture reads the uv (only image textures do;
// the reference computes it on every sphere hit, sphere.cuh:141-150, to the same values).  Float
// acos/atan2 for the nvcc flavour, double-evaluated for the g++ flavour (closest to glibc).
template <bool FLOAT_TRIG>
__device__ __forceinline__ void hit_uv(const DevScene& S, Hit& h, V3 outward) {
    h.sphere_uv = false;
    float theta, phi;
    if (FLOAT_TRIG) {
        theta = acosf(-outward.y);
        phi = atan2f(-outward.z, outward.x) + 3.14159265358979323846f;
    } else {
        theta = (float)acos((double)(-outward.y));
        phi = (float)atan2((double)(-outward.z), (double)outward.x) + 3.14159265358979323846f;
    }
    float sc = phi / (2.0f * 3.14159265358979323846f);
    float tc = theta / 3.14159265358979323846f;
    sc = fmod1(sc * 1.0f);
    tc = fmod1(tc * 1.0f);
    h.u = 1.0f * sc + 0.0f;
    h.v = 1.0f * tc + 0.0f;
}
// The pending uv of a world-space sphere hit: its outward normal again, (p - c) / r with the same
// operands and roundings as finalize_prim's.
template <bool FLOAT_TRIG>
__device__ __forceinline__ void hit_uv(const DevScene& S, Hit& h) {
    if (!h.sphere_uv) return;
    const float4 s = __ldg(S.sph + (h.item & ITEM_INDEX_MASK));
    hit_uv<FLOAT_TRIG>(S, h, divs(sub(h.p, v3(s.x, s.y, s.z)), s.w));
}

template <bool FLOAT_TRIG, bool EAGER_UV = false>
__device__ __forceinline__ void finalize_prim(const DevScene& S, uint32_t kind, uint32_t idx, float t, V3 o, V3 d,
                                              Hit& h) {
    switch (kind) {
    case ITEM_SPHERE: {
        float4 s = __ldg(S.sph + idx);
        h.p = at(o, d, t);
        h.mat = __ldg(S.sph_aux + idx).x;
        V3 c = v3(s.x, s.y, s.z);
        V3 outward = divs(sub(h.p, c), s.w);
        set_face_normal(h, d, outward);
        // the uv (get_sphere_uv) only feeds image textures: a hit in world space computes it when a
        // texture reads it (hit_uv, from the same hit point and record); a transformed sphere's hit
        // (object space here) computes it now
        h.sphere_uv = true;
        if (EAGER_UV) hit_uv<FLOAT_TRIG>(S, h, outward);
    } break;
    case ITEM_QUAD:
    case ITEM_LIGHT: {
        const float4* q = kind == ITEM_QUAD ? S.quad + 5 * (size_t)idx : S.light + 6 * (size_t)idx;
        float4 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3), q4 = __ldg(q + 4);
        if (kind == ITEM_LIGHT && q4.w < 0.0f) {
            // omni / spot light (omni_light.cuh:85-102): outward normal (p - c) / radius; its texture is
            // a solid colour, so the sphere uv the reference also computes is not needed
            h.p = at(o, d, t);
            h.mat = __float_as_int(q1.w);
            set_face_normal(h, d, divs(sub(h.p, v3(q0.x, q0.y, q0.z)), q0.w));
            h.u = 0.0f;
            h.v = 0.0f;
            break;
        }
        V3 n = v3(q0.x, q0.y, q0.z);
        V3 ip = at(o, d, t);
        V3 pl = sub(ip, v3(q1.x, q1.y, q1.z));
        V3 w = v3(q4.x, q4.y, q4.z);
        float a = dot(w, cross(pl, v3(q3.x, q3.y, q3.z)));
        float b = dot(w, cross(v3(q2.x, q2.y, q2.z), pl));
        h.p = ip;
        h.mat = __float_as_int(q1.w);
        set_face_normal(h, d, n);
        if (kind == ITEM_QUAD) { h.u = a; h.v = b; }
        else { h.u = a + 0.5f; h.v = b + 0.5f; }
    } break;
    default: {  // triangle
        const float4* p = S.tri + 3 * (size_t)idx;
        float4 a0 = __ldg(p), a1 = __ldg(p + 1), a2 = __ldg(p + 2);
        h.p = at(o, d, t);
        h.mat = __float_as_int(a0.w);
        float4 nn = __ldg(S.tri_n + idx);
        V3 normal = v3(nn.x, nn.y, nn.z);
        int sm = __float_as_int(a2.w);
        if (sm >= 0) {
            // smooth: a*vn1 + b*vn2 + c*vn0 with the barycentrics of triangle::hit (triangle.cuh:171-175)
            V3 v0 = v3(a0.x, a0.y, a0.z), e1 = v3(a1.x, a1.y, a1.z), e2 = v3(a2.x, a2.y, a2.z);
            V3 pv = cross(d, e2);
            float det = dot(e1, pv);
            float inv_det = 1.0f / det;
            V3 tv = sub(o, v0);
            float bu = dot(tv, pv) * inv_det;
            V3 qv = cross(tv, e1);
            float bv = dot(d, qv) * inv_det;
            float bc = 1.0f - bu - bv;
            const float4* vn = S.tri_vn + 3 * (size_t)sm;
            normal = add(add(mul(bu, v3(__ldg(vn + 1))), mul(bv, v3(__ldg(vn + 2)))), mul(bc, v3(__ldg(vn))));
        }
        set_face_normal(h, d, normal);
        if (S.tri_uv) {
            tri_uv_at(S, idx, a0, a1, a2, h);
        } else {
            // no mesh has texture coordinates: get_triangle_uv over all-zero vertex uvs gives (0, 0)
            h.u = 0.0f;
            h.v = 0.0f;
        }
    } break;
    }
}

// A box face (aarect.cuh hit()): hit point r.at(t), the axis normal (negated by rt::flip_normals for the
// low faces), front_face left at hit_record's default true, uv by get_xy/xz/yz_rect_uv with the default
// mapping.
__device__ __forceinline__ void finalize_rect(const DevScene& S, uint32_t idx, float t, V3 o, V3 d, Hit& h) {
    const float4 r0 = __ldg(S.rect + 2 * (size_t)idx), r1 = __ldg(S.rect + 2 * (size_t)idx + 1);
    const int axis = __float_as_int(r1.y);
    const float o0 = axis == 2 ? o.y : o.x, d0 = axis == 2 ? d.y : d.x;
    const float o1 = axis == 0 ? o.y : o.z, d1 = axis == 0 ? d.y : d.z;
    const float a = o0 + t * d0, b = o1 + t * d1;
    float su = (a - r0.x) / (r0.y - r0.x);
    float sv = (b - r0.z) / (r0.w - r0.z);
    su = fmod1(su * 1.0f);
    sv = fmod1(sv * 1.0f);
    h.u = 1.0f * su + 0.0f;
    h.v = 1.0f * sv + 0.0f;
    h.p = at(o, d, t);
    const float sgn = r1.z != 0.0f ? -1.0f : 1.0f;
    h.n = axis == 0 ? v3(0.0f, 0.0f, sgn) : axis == 1 ? v3(0.0f, sgn, 0.0f) : v3(sgn, 0.0f, 0.0f);
    h.front = true;
    h.mat = __float_as_int(r1.w);
}

template <bool FLOAT_TRIG>
__device__ __forceinline__ void finalize_hit(const DevScene& S, uint32_t it, float t, V3 o, V3 d, Hit& h) {
    const uint32_t kind = it >> ITEM_KIND_SHIFT, idx = it & ITEM_INDEX_MASK;
    h.t = t;
    h.item = it;
    h.sphere_uv = false;
#if !RTC_XP
    // only the RTC_XP=1 kernels walk the xprim BVH, so an item here is always a plain primitive; keeping
    // the xprim branch out of these kernels keeps its registers out of the shade kernel
    finalize_prim<FLOAT_TRIG>(S, kind, idx, t, o, d, h);
#else
    if (kind != ITEM_XPRIM) {
        finalize_prim<FLOAT_TRIG>(S, kind, idx, t, o, d, h);
        return;
    }
    // a transformed primitive or a box face: the inner hit in object space, then back to world space
    const int4 x = __ldg(S.xprim + idx);
    if (x.x >= 0) xf_to_object(S, x.x, o, d);
    if (x.y == XPRIM_RECT) finalize_rect(S, (uint32_t)x.z, t, o, d, h);
    else finalize_prim<FLOAT_TRIG, true>(S, (uint32_t)x.y, (uint32_t)x.z, t, o, d, h);
    if (x.x >= 0) xf_to_world(S, x.x, h.p, h.n);
#endif
}

// ------------------------------------------------------------------------------------------------
// textures and materials
// ------------------------------------------------------------------------------------------------
struct RGB {
    float r, g, b;
};
__device__ __forceinline__ RGB rgb(float r, float g, float b) { RGB c; c.r = r; c.g = g; c.b = b; return c; }

// texture::value dispatch: solid (solid_color_texture.cuh:34), checker (checker_texture.cuh:33-41),
// image (image_texture.cuh:54-70 + bitmap_image::pixel_data, bitmap_image.cuh:74-91).
template <bool FLOAT_TRIG>
__device__ __forceinline__ RGB texture_value(const DevScene& S, int tex, Hit& h, uint32_t& status) {
    const V3 p = h.p;
    for (int guard = 0; guard < 8; ++guard) {
        if ((uint32_t)tex >= S.num_textures) { status |= STATUS_BAD_TEXTURE; return rgb(0.f, 0.f, 0.f); }
        int4 ti = __ldg(S.tex_i + tex);
        float4 tf = __ldg(S.tex_f + tex);
        if (ti.x == 0) return rgb(tf.x, tf.y, tf.z);
        if (ti.x == 1) {
            int xi = (int)floorf(tf.w * p.x);
            int yi = (int)floorf(tf.w * p.y);
            int zi = (int)floorf(tf.w * p.z);
            bool even = (xi + yi + zi) % 2 == 0;   // C++ remainder: odd negative sums give -1
            tex = even ? ti.y : ti.z;
            continue;
        }
        // image
        if ((uint32_t)ti.w >= S.num_images) { status |= STATUS_BAD_TEXTURE; return rgb(0.f, 0.f, 0.f); }
        int4 im = __ldg(S.images + ti.w);
        int W = im.y, H = im.z;
        if (H <= 0) return rgb(0.f, 1.f, 1.f);
        hit_uv<FLOAT_TRIG>(S, h);
        const float u = h.u, v = h.v;
        float uu = u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
        float vc = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
        float vv = 1.0f - vc;
        int i = (int)(uu * (float)W);
        int j = (int)(vv * (float)H);
        i = i < 0 ? 0 : (i < W ? i : W - 1);
        j = j < 0 ? 0 : (j < H ? j : H - 1);
        const uint8_t* px = S.image_bytes + (size_t)im.x + (size_t)j * (size_t)(W * 3) + (size_t)i * 3;
        const float cs = 1.0f / 255.0f;
        return rgb(cs * (float)px[0], cs * (float)px[1], cs * (float)px[2]);
    }
    status |= STATUS_BAD_TEXTURE;
    return rgb(0.f, 0.f, 0.f);
}

// background colour of a missed ray (camera.cuh:161-174)
__device__ __forceinline__ RGB background(const DevScene& S, V3 dir) {
    const DevBackground& B = S.bg;
    if (B.kind == 0) return rgb(B.color[0], B.color[1], B.color[2]);
    V3 ud = unit(dir);
    if (B.kind == 1) {
        float a = 0.5f * (ud.y + 1.0f);
        float b = 1.0f - a;
        return rgb(b * B.color[0] + a * B.top[0], b * B.color[1] + a * B.top[1], b * B.color[2] + a * B.top[2]);
    }
    double theta = acos((double)-ud.y);
    double phi = atan2((double)-ud.z, (double)ud.x) + 3.14159265358979323846;
    double uu = phi / (2.0 * 3.14159265358979323846);
    double vv = theta / 3.14159265358979323846;
    int W = B.env_w, H = B.env_h;
    int x = (int)(uu * W);
    x = x < 0 ? 0 : (x >= W ? W - 1 : x);
    int y = (int)((1.0 - vv) * H);
    y = y < 0 ? 0 : (y >= H ? H - 1 : y);
    const float* px = B.env + 3 * ((size_t)y * W + x);
    return rgb(__ldg(px), __ldg(px + 1), __ldg(px + 2));
}

// ---- environment-map importance sampling (clean mode, RTC_FLAG_ENV_SAMPLING) ---------------------
// The distribution of image_pdf (pdf/image_pdf.cuh:32-145) done so that generate and value agree: a row
// by the marginal CDF, a column by the row's conditional CDF (each by binary search, the CDFs inverted
// continuously so the point is uniform inside its texel), the point (u, v) turned into a direction by
// from_spherical_uv (uvmapping.cuh:194-200), whose inverse is the background lookup above
// (get_spherical_uv, uvmapping.cuh:144-158).  Density over directions: texel probability x W x H /
// (2 pi^2 sin(theta)).

// first index in cdf[0, n) whose value exceeds r (n - 1 at most)
__device__ __forceinline__ int env_search(const float* cdf, int n, float r) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) > r) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ V3 env_sample(const DevBackground& B, float r1, float r2) {
    const int W = B.env_w, H = B.env_h;
    const int y = env_search(B.cdf, H, r1);
    const float m0 = y > 0 ? __ldg(B.cdf + y - 1) : 0.0f, m1 = __ldg(B.cdf + y);
    const float fy = m1 > m0 ? fminf(fmaxf((r1 - m0) / (m1 - m0), 0.0f), 1.0f) : 0.5f;
    const float* C = B.cdf + H + (size_t)y * W;
    const int x = env_search(C, W, r2);
    const float c0 = x > 0 ? __ldg(C + x - 1) : 0.0f, c1 = __ldg(C + x);
    const float fx = c1 > c0 ? fminf(fmaxf((r2 - c0) / (c1 - c0), 0.0f), 1.0f) : 0.5f;
    const float u = ((float)x + fx) / (float)W;
    const float v = 1.0f - ((float)y + fy) / (float)H;
    float st, ct, sa, ca;
    sincosf(3.14159265358979323846f * v, &st, &ct);
    sincosf(2.0f * 3.14159265358979323846f * u - 3.14159265358979323846f, &sa, &ca);
    return v3(st * ca, -ct, -st * sa);
}

__device__ __forceinline__ float env_pdf(const DevBackground& B, V3 dir) {
    const V3 ud = unit(dir);
    const double theta = acos((double)-ud.y);
    const double phi = atan2((double)-ud.z, (double)ud.x) + 3.14159265358979323846;
    const int W = B.env_w, H = B.env_h;
    int x = (int)(phi / (2.0 * 3.14159265358979323846) * W);
    x = x < 0 ? 0 : (x >= W ? W - 1 : x);
    int y = (int)((1.0 - theta / 3.14159265358979323846) * H);
    y = y < 0 ? 0 : (y >= H ? H - 1 : y);
    const float* C = B.cdf + H + (size_t)y * W;
    const float pr = __ldg(B.cdf + y) - (y > 0 ? __ldg(B.cdf + y - 1) : 0.0f);
    const float pc = __ldg(C + x) - (x > 0 ? __ldg(C + x - 1) : 0.0f);
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ud.y * ud.y));
    return st > 0.0f ? pr * pc * B.pdf_scale / st : 0.0f;
}

// directional_light::pdf_value (directional_light.cuh:147-158) for light `li` seen from o along v;
// omni_light::pdf_value / spot_light::pdf_value (omni_light.cuh:104-115): 1 / the solid angle of the
// sphere, 2 * M_PI * (1 - cos_theta_max), all in float: the reference's M_PI is a float literal
// (misc/constants.cuh:35).
__device__ __forceinline__ float light_pdf_value(const DevScene& S, uint32_t li, V3 o, V3 v) {
    const float4* q = S.light + 6 * (size_t)li;
    float4 q0 = __ldg(q), q4 = __ldg(q + 4);
    float t, a, b;
    if (q4.w < 0.0f) {
        if (!sphere_t(q0, o, v, 0.00001f, INFINITY, t)) return 0.0f;
        const float ctm = sqrtf(1.0f - q0.w * q0.w / lensq(sub(v3(q0.x, q0.y, q0.z), o)));
        const float solid_angle = 2.0f * 3.14159265358979323846f * (1.0f - ctm);
        return 1.0f / solid_angle;
    }
    if (!planar_t(q0, __ldg(q + 1), __ldg(q + 2), __ldg(q + 3), q4, o, v, 0.00001f, INFINITY, true, t, a, b)) return 0.0f;
    V3 n = v3(q0.x, q0.y, q0.z);
    V3 nrm = dot(v, n) < 0.0f ? n : neg(n);
    float distance_squared = t * t * lensq(v);
    float cosine = fabsf(dot(v, nrm) / len(v));
    return distance_squared / (cosine * q4.w);
}

// hittable_list::pdf_value over the light list (hittable_list.cuh:173-184)
__device__ __forceinline__ float lights_pdf_value(const DevScene& S, V3 o, V3 v) {
    float weight = 1.0f / (float)S.num_lights;
    float sum = 0.0f;
    for (uint32_t i = 0; i < S.num_lights; ++i) sum += weight * light_pdf_value(S, i, o, v);
    return sum;
}

// prepare_pixel_color (color.cuh:289-309) and the output loop (gpu.cu:792-799, 2098-2107) for one pixel:
// NaN -> 0, * (1/spp), sqrt, int(255.99 * clamp(c, 0, 0.999)), written to the row-flipped RGB8 image.
// `p` is the frame-buffer index j*W + i with j counted from the bottom.
__device__ __forceinline__ void quantize_pixel(float4 c, int spp, int width, int height, int64_t p, uint8_t* rgb8) {
    const int i = (int)(p % width), j = (int)(p / width);
    const float ch[3] = {c.x, c.y, c.z};
    uint8_t* o = rgb8 + ((size_t)(height - j - 1) * width + i) * 3;
    for (int k = 0; k < 3; ++k) {
        float x = ch[k] != ch[k] ? 0.0f : ch[k];
        if (spp > 0) x *= 1.0f / (float)spp;
        x = sqrtf(x);
        const float cl = x < 0.0f ? 0.0f : (x > 0.999f ? 0.999f : x);
        o[k] = (uint8_t)(int)(255.99f * cl);
    }
}

}  // namespace RTC_XP_NS
}  // namespace rtc
