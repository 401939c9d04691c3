// rtc_path.cuh - camera rays and the per-sample path loop.
//
// Compat mode restates camera::ray_color (core/src/cameras/camera.cuh:149-264) with the reference's
// materials and PDFs, consuming one thrust::minstd_rand stream per pixel in the reference's order.
// Clean mode keeps the same materials but draws from a counter-based stream per (pixel, sample),
// samples the light list only when it is non-empty, and traces spp samples.
#pragma once

#include "rtc_trace.cuh"

namespace rtc {
inline namespace RTC_XP_NS {

// Multi-draw expressions: the reference builds vectors from several get_real() calls inside one
// constructor call or overloaded-operator expression, whose evaluation order C++ leaves open.
// ORDER 0 consumes them left to right (nvcc device build), ORDER 1 right to left (g++ build).
template <int ORDER, class R>
__device__ __forceinline__ void draw2(R& rng, float& first_arg, float& second_arg) {
    if (ORDER == 0) { first_arg = rng.uniform(); second_arg = rng.uniform(); }
    else { second_arg = rng.uniform(); first_arg = rng.uniform(); }
}
template <int ORDER, class R>
__device__ __forceinline__ void draw3(R& rng, float& a, float& b, float& c) {
    if (ORDER == 0) { a = rng.uniform(); b = rng.uniform(); c = rng.uniform(); }
    else { c = rng.uniform(); b = rng.uniform(); a = rng.uniform(); }
}

// random_in_unit_disk (gpu_randomizer.cuh:61-67)
//
// ORDER 0 (the builds with FMA contraction: the nvcc flavour and clean mode) writes the camera
// sample's multiply-adds as explicit fused operations, so its rounding is fixed by the source and not
// by how the compiler contracts the kernel that inlines it: a pixel's camera rays are the same bits
// whichever kernel (admission, shade, drain) starts its sample.
template <int ORDER, class R>
__device__ __forceinline__ V3 random_in_unit_disk(R& rng) {
    V3 p;
    do {
        float a, b;
        draw2<ORDER>(rng, a, b);
        p = v3(2.0f * a - 1.0f, 2.0f * b - 1.0f, 2.0f * 0.0f - 0.0f);   // 2*a is exact: fused or not
    } while ((ORDER == 0 ? __fmaf_rn(p.x, p.x, __fmaf_rn(p.y, p.y, __fmul_rn(p.z, p.z))) : dot(p, p)) >= 1.0f);
    return p;
}

// random_in_unit_sphere (gpu_randomizer.cuh:70-76); l1() is the squared length (vector3.cuh:86-88)
template <int ORDER, class R>
__device__ __forceinline__ V3 random_in_unit_sphere(R& rng) {
    V3 p;
    do {
        float a, b, c;
        draw3<ORDER>(rng, a, b, c);
        p = v3(2.0f * a - 1.0f, 2.0f * b - 1.0f, 2.0f * c - 1.0f);
    } while (p.x * p.x + p.y * p.y + p.z * p.z >= 1.0f);
    return p;
}

// Transcendentals follow the reference build being reproduced.  FLOAT_TRIG (the nvcc flavour and
// clean mode): CUDA's float functions, as the reference's device build calls them.  Otherwise (the g++
// flavour): evaluated in double and rounded, which agrees with glibc's cosf/sinf on ~98.7% of inputs
// and is within 1 ulp otherwise.
template <bool FLOAT_TRIG>
__device__ __forceinline__ void cos_sin(float phi, float& c, float& s) {
    if (FLOAT_TRIG) {
        sincosf(phi, &s, &c);
    } else {
        double sd, cd;
        sincos((double)phi, &sd, &cd);
        c = (float)cd;
        s = (float)sd;
    }
}

// random_cosine_direction (gpu_randomizer.cuh:121-133)
template <bool FLOAT_TRIG, class R>
__device__ __forceinline__ V3 random_cosine_direction(R& rng) {
    const float r1 = rng.uniform();
    const float r2 = rng.uniform();
    const float phi = 6.28318530718f * r1;
    const float z = sqrtf(1.0f - r2);
    const float r2s = sqrtf(r2);
    float c, s;
    cos_sin<FLOAT_TRIG>(phi, c, s);
    return v3(c * r2s, s * r2s, z);
}

// onb::build_from_w (onb.cuh:122-128)
struct Onb {
    V3 u, v, w;
};
__device__ __forceinline__ Onb build_from_w(V3 n) {
    Onb b;
    b.w = unit(n);
    V3 a = (fabsf(b.w.x) > 0.9f) ? v3(0.f, 1.f, 0.f) : v3(1.f, 0.f, 0.f);
    b.v = unit(cross(b.w, a));
    b.u = cross(b.w, b.v);
    return b;
}
// onb::local (onb.cuh:117-120): a.x*u + a.y*v + a.z*w
__device__ __forceinline__ V3 onb_local(const Onb& b, V3 a) {
    return add(add(mul(a.x, b.u), mul(a.y, b.v)), mul(a.z, b.w));
}

// random_to_sphere (gpu_randomizer.cuh:82-93): z = 1 + r2 (sqrt(1 - R^2/d^2) - 1), phi = 2 M_PI r1 in float
// (the reference's M_PI is a float literal, misc/constants.cuh:35), x = cos(phi) sqrt(1 - z^2),
// y = sin(phi) sqrt(1 - z^2).
template <bool FLOAT_TRIG, class R>
__device__ __forceinline__ V3 random_to_sphere(R& rng, float radius, float distance_squared) {
    const float r1 = rng.uniform();
    const float r2 = rng.uniform();
    const float z = 1.0f + r2 * (sqrtf(1.0f - radius * radius / distance_squared) - 1.0f);
    const float phi = 2.0f * 3.14159265358979323846f * r1;
    float c, s;
    cos_sin<FLOAT_TRIG>(phi, c, s);
    return v3(c * sqrtf(1.0f - z * z), s * sqrtf(1.0f - z * z), z);
}

// directional_light::random (directional_light.cuh:165-171): P + (U-0.5)*u + (U-0.5)*v - o; for omni
// and spot lights omni_light::random (omni_light.cuh:117-124): onb(center - o).local(random_to_sphere).
template <int ORDER, class R>
__device__ __forceinline__ V3 light_random(const DevScene& S, uint32_t li, V3 o, R& rng) {
    const float4* q = S.light + 6 * (size_t)li;
    if (__ldg(q + 4).w < 0.0f) {
        const float4 c = __ldg(q);
        const V3 dir = sub(v3(c.x, c.y, c.z), o);
        const Onb b = build_from_w(dir);
        return onb_local(b, random_to_sphere<ORDER == 0>(rng, c.w, lensq(dir)));
    }
    float4 P = __ldg(q + 1), U = __ldg(q + 2), Vv = __ldg(q + 3);
    float ru, rv;
    draw2<ORDER>(rng, ru, rv);
    V3 p = add(add(v3(P.x, P.y, P.z), mul(ru - 0.5f, v3(U.x, U.y, U.z))), mul(rv - 0.5f, v3(Vv.x, Vv.y, Vv.z)));
    return sub(p, o);
}

struct Ray {
    V3 o, d;
    float time;
};

// perspective_camera::get_ray (perspective_camera.cuh:112-117): the disk sample and the time sample
// are drawn even when the aperture is zero.
template <int ORDER, class R>
__device__ __forceinline__ Ray camera_ray(const DevCamera& c, float s, float t, R& rng) {
    V3 rd = mul(c.lens_radius, random_in_unit_disk<ORDER>(rng));
    Ray r;
    if constexpr (ORDER == 0) {
        // fused multiply-adds spelled out (see random_in_unit_disk)
        float off[3], o[3], d[3];
        for (int k = 0; k < 3; ++k) off[k] = __fmaf_rn(c.v[k], rd.y, __fmul_rn(c.u[k], rd.x));
        float time = __fmaf_rn(rng.uniform(), __fsub_rn(c.time1, c.time0), c.time0);
        for (int k = 0; k < 3; ++k) {
            o[k] = __fadd_rn(c.origin[k], off[k]);
            d[k] = __fsub_rn(__fsub_rn(__fmaf_rn(t, c.vertical[k], __fmaf_rn(s, c.horizontal[k], c.llc[k])), c.origin[k]),
                             off[k]);
        }
        r.o = v3(o[0], o[1], o[2]);
        r.d = v3(d[0], d[1], d[2]);
        r.time = time;
    } else {
        V3 offset = add(mul(v3(c.u), rd.x), mul(v3(c.v), rd.y));
        float time = c.time0 + rng.uniform() * (c.time1 - c.time0);
        r.o = add(v3(c.origin), offset);
        r.d = sub(sub(add(add(v3(c.llc), mul(s, v3(c.horizontal))), mul(t, v3(c.vertical))), v3(c.origin)), offset);
        r.time = time;
    }
    return r;
}

// Clean mode starts scattered rays from a point pushed off the surface along the normal of the side
// the new ray leaves from: Waechter & Binder, "A Fast and Robust Method for Avoiding Self-Intersection",
// Ray Tracing Gems (2019), ch. 6.  The offset is a fixed number of ulps of each coordinate (a fixed
// distance near the origin), so whether the next ray re-hits its own surface no longer depends on
// last-bit rounding.  Compat mode keeps the reference's start point and tmin = 1e-5 (constants.cuh:27).
__device__ __forceinline__ float offset_coord(float p, float n) {
    const float kOrigin = 1.0f / 32.0f, kFloatScale = 1.0f / 65536.0f, kIntScale = 256.0f;
    const int of = (int)(kIntScale * n);
    const float pi = __int_as_float(__float_as_int(p) + (p < 0.0f ? -of : of));
    return fabsf(p) < kOrigin ? p + kFloatScale * n : pi;
}
template <bool CLEAN>
__device__ __forceinline__ V3 scatter_origin(V3 p, V3 n, V3 dir) {
    if (!CLEAN) return p;
    const V3 side = dot(dir, n) < 0.0f ? neg(n) : n;
    return v3(offset_coord(p.x, side.x), offset_coord(p.y, side.y), offset_coord(p.z, side.z));
}

struct PathCounters {
    uint32_t rays, nodes, prims;
};

// material::scatter of the hit material (metal, dielectric or lambertian; lights are handled by the
// caller): updates the attenuation and turns `r` into the scattered ray (camera.cuh:185-225).
template <bool CLEAN, int ORDER, class R>
__device__ __forceinline__ void scatter_bounce(const DevScene& S, Ray& r, Hit& h, int4 mi, float4 mf, RGB& att,
                                               R& rng, uint32_t& status) {
    constexpr bool FT = CLEAN || ORDER == 0;   // float trig in the nvcc flavour and in clean mode
    if (mi.x == 1) {
        // metal::scatter (metal.cuh:57-64)
        RGB a = texture_value<FT>(S, mi.y, h, status);
        V3 refl = reflect(unit(r.d), h.n);
        V3 rs = random_in_unit_sphere<ORDER>(rng);
        r.d = add(refl, mul(mf.x, rs));
        r.o = scatter_origin<CLEAN>(h.p, h.n, r.d);
        att.r *= a.r;
        att.g *= a.g;
        att.b *= a.b;
        return;
    }
    if (mi.x == 2) {
        // dielectric::scatter (dielectric.cuh:32-52) with Schlick (dielectric.cuh:57-63)
        float ratio = h.front ? (1.0f / mf.y) : mf.y;
        V3 ud = unit(r.d);
        float ct = dot(neg(ud), h.n);
        float cos_theta = ct < 1.0f ? ct : 1.0f;
        float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
        bool cannot_refract = ratio * sin_theta > 1.0f;
        bool do_reflect = cannot_refract;
        if (!cannot_refract) {
            float r0 = (1.0f - ratio) / (1.0f + ratio);
            r0 = r0 * r0;
            // (float)pow(1 - cosine, 5): the x^5 product in double agrees with glibc's double pow
            double x = (double)(1.0f - cos_theta);
            double x2 = x * x;
            float p5 = (float)(x2 * x2 * x);
            float refl = r0 + (1.0f - r0) * p5;
            do_reflect = refl > rng.uniform();
        }
        r.d = do_reflect ? reflect(ud, h.n) : refract(ud, h.n, ratio);
        r.o = scatter_origin<CLEAN>(h.p, h.n, r.d);
        return;   // attenuation (1,1,1)
    }
    // lambertian::scatter (lambertian.cuh:63-131): attenuation from the texture, cosine_pdf(normal)
    RGB a = texture_value<FT>(S, mi.y, h, status);
    Onb b = build_from_w(h.n);
    V3 dir;
    float pdf_val, spdf;
    if (CLEAN && S.bg.cdf) {
        // with environment-map sampling: mixture_pdf(objects, background, 0.8) (camera.cuh:333-336),
        // objects = the light/cosine mixture below (cosine alone without lights)
        const bool lights = S.num_lights > 0;
        const float pick = rng.uniform();
        if (pick < 0.2f) {
            const float r1 = rng.uniform(), r2 = rng.uniform();
            dir = env_sample(S.bg, r1, r2);
        } else if (lights && rng.uniform() < 0.5f) {
            if (S.num_lights > 1) (void)rng.uniform();
            dir = light_random<ORDER>(S, 0, h.p, rng);
        } else {
            dir = onb_local(b, random_cosine_direction<FT>(rng));
        }
        float cosv = dot(unit(dir), b.w) / 3.14159265358979323846f;
        float cpdf = 0.0f > cosv ? 0.0f : cosv;
        const float obj = lights ? 0.5f * lights_pdf_value(S, h.p, dir) + 0.5f * cpdf : cpdf;
        pdf_val = 0.8f * obj + 0.2f * env_pdf(S.bg, dir);
    } else if (!CLEAN || S.num_lights > 0) {
        // mixture_pdf(hittable_pdf(lights, p), cosine_pdf), proportion 0.5 (mixture_pdf.cuh:28-47)
        if (rng.uniform() < 0.5f) {
            if (S.num_lights == 0) {
                dir = v3(0.f, 0.f, 0.f);   // hittable_list::random on an empty list
            } else {
                if (S.num_lights > 1) (void)rng.uniform();   // get_int(rng, 0, n-1) == 0, one draw
                dir = light_random<ORDER>(S, 0, h.p, rng);
            }
        } else {
            dir = onb_local(b, random_cosine_direction<FT>(rng));
        }
        float cosv = dot(unit(dir), b.w) / 3.14159265358979323846f;
        float cpdf = 0.0f > cosv ? 0.0f : cosv;   // ffmax(0, x) keeps NaN
        pdf_val = 0.5f * lights_pdf_value(S, h.p, dir) + (1.0f - 0.5f) * cpdf;
    } else {
        dir = onb_local(b, random_cosine_direction<FT>(rng));
        float cosv = dot(unit(dir), b.w) / 3.14159265358979323846f;
        pdf_val = 0.0f > cosv ? 0.0f : cosv;
    }
    // lambertian::scattering_pdf (lambertian.cuh:139-143)
    float cos_theta = dot(h.n, unit(dir));
    spdf = cos_theta < 0.0f ? 0.0f : cos_theta / 3.14159265358979323846f;
    // current_attenuation *= srec.attenuation * scattering_pdf / pdf_val, where color / t = (1/t) * color
    float rcp = 1.0f / pdf_val;
    att.r *= rcp * (a.r * spdf);
    att.g *= rcp * (a.g * spdf);
    att.b *= rcp * (a.b * spdf);
    r.o = scatter_origin<CLEAN>(h.p, h.n, dir);
    r.d = dir;
}

__device__ __forceinline__ bool is_light_material(int kind) { return kind == 3 || kind == MAT_SPOT_LIGHT; }

// material::emitted of the hit (diffuse_light.cuh:45-67, diffuse_spot_light.cuh:33-49; other materials
// emit (0,0,0)).  `alpha0` is set for an emission with alpha 0 - the back face of a one-sided light -
// which makes camera::ray_color re-hit the scene from just behind it (camera.cuh:177-183).
template <bool FT>
__device__ __forceinline__ RGB emitted(const DevScene& S, const Ray& r, Hit& h, int4 mi, float4 mf, bool& alpha0,
                                       uint32_t& status) {
    RGB em = rgb(0.f, 0.f, 0.f);
    alpha0 = false;
    if (mi.x == 3) {
        if (mf.w != 0.0f && !h.front) {
            alpha0 = true;   // RGBA(0,0,0,0): back face of a one-sided light
        } else {
            RGB tv = texture_value<FT>(S, mi.y, h, status);
            em = rgb(tv.r * mf.z, tv.g * mf.z, tv.b * mf.z);
        }
    } else if (mi.x == MAT_SPOT_LIGHT) {
        // diffuse_spot_light::emitted (diffuse_spot_light.cuh:33-49).  Back face: RGBA(0,0,0,0) when
        // invisible, else RGBA(1,1,1,0) (both re-hit; the product with the attenuation adds 0 or 1);
        // outside the cone RGBA(1,1,1,1); inside texture * (intensity * pow(cos, falloff)).
        const float4* q = S.light + 6 * (size_t)mi.z;
        const float4 sd = __ldg(q + 2), cone = __ldg(q + 3);
        if (!h.front) {
            alpha0 = true;
            if (cone.w == 0.0f) em = rgb(1.f, 1.f, 1.f);
        } else {
            const float cos_theta = dot(unit(r.d), unit(v3(sd.x, sd.y, sd.z)));
            if (cos_theta < cone.x) {
                em = rgb(1.f, 1.f, 1.f);
            } else {
                const float attn = FT ? powf(cos_theta, cone.y) : (float)pow((double)cos_theta, (double)cone.y);
                const float k = mf.z * attn;
                RGB tv = texture_value<FT>(S, mi.y, h, status);
                em = rgb(tv.r * k, tv.g * k, tv.b * k);
            }
        }
    }
    return em;
}

// One bounce of camera::ray_color (camera.cuh:153-227) AFTER the closest-hit query of the current ray:
// `hit` tells whether world.hit found something at (t, item).  Updates the path's running radiance
// `result`, its attenuation `att` and its ray.  All additions of the reference are kept, including the
// zero emission of non-emitting materials, so NaN/Inf propagate exactly as in the reference.  The
// "invisible" re-hit from behind a one-sided light (camera.cuh:177-183) is handed back to the caller
// instead of traced here, so every engine has one trace call site: the wavefront sends the re-hit
// through its extend kernel like any other ray, the megakernel and the drain loop around (trace_bounces).
//   BOUNCE_END    the path ends at this bounce;
//   BOUNCE_NEXT   the path continues with the scattered ray (one depth level used);
//   BOUNCE_REHIT  the hit was the back face of a one-sided light: its (zero-alpha) emission is added
//                 and the same ray must be traced again from `rehit_tmin` = t + 0.001, at the same
//                 depth; the next call passes `rehit` = true with that trace's result.
// With `rehit`, a miss or a light leaves the path ending on the light (rec keeps the light's material,
// whose scatter returns false), anything else scatters with no emission added - exactly camera.cuh:177-190.
enum BounceOut { BOUNCE_END = 0, BOUNCE_NEXT = 1, BOUNCE_REHIT = 2 };
template <bool CLEAN, int ORDER, class R>
__device__ __forceinline__ int shade_bounce_deferred(const DevScene& S, Ray& r, bool hit, float t, uint32_t item,
                                                     bool rehit, RGB& result, RGB& att, R& rng, uint32_t& status,
                                                     float& rehit_tmin) {
    constexpr bool FT = CLEAN || ORDER == 0;
    if (!hit) {
        if (rehit) return BOUNCE_END;
        RGB bg = background(S, r.d);
        result.r += att.r * bg.r;
        result.g += att.g * bg.g;
        result.b += att.b * bg.b;
        return BOUNCE_END;
    }
    Hit h;
    finalize_hit<FT>(S, item, t, r.o, r.d, h);
    if ((uint32_t)h.mat >= S.num_materials) { status |= STATUS_BAD_MATERIAL; return BOUNCE_END; }
    const int4 mi = __ldg(S.mat_i + h.mat);
    const float4 mf = __ldg(S.mat_f + h.mat);
    if (!rehit) {
        bool em_alpha0;
        const RGB em = emitted<FT>(S, r, h, mi, mf, em_alpha0, status);
        result.r += att.r * em.r;
        result.g += att.g * em.g;
        result.b += att.b * em.b;
        if (em_alpha0) {
            rehit_tmin = h.t + 0.001f;
            return BOUNCE_REHIT;
        }
    }
    if (is_light_material(mi.x)) return BOUNCE_END;
    scatter_bounce<CLEAN, ORDER>(S, r, h, mi, mf, att, rng, status);
    return BOUNCE_NEXT;
}

// camera::ray_color's loop (camera.cuh:155-226) from `depth` levels left down to the end of the path:
// trace, then shade; a re-hit from behind a one-sided light traces the same ray again from `tmin` =
// t + 0.001 at the same depth.  `tmin` starts at 1e-5 (SHADOW_ACNE_FIX), or at a pending re-hit's start.
template <bool CLEAN, int ORDER, class R>
__device__ __forceinline__ void trace_bounces(const DevScene& S, Ray& r, int depth, int max_depth, float tmin,
                                              RGB& result, RGB& att, R& rng, PathCounters& pc, TraceStats& st,
                                              uint32_t& status) {
    bool rehit = tmin > 0.00001f;
    for (; depth > 0; --depth) {
        const bool hide = depth == max_depth;
        float t, next_tmin = 0.0f;
        uint32_t item;
        pc.rays++;
        const bool hit = closest_hit<CLEAN>(S, r.o, r.d, tmin, 3.402823466e+38f, hide, t, item, st, status);
        const int out = shade_bounce_deferred<CLEAN, ORDER>(S, r, hit, t, item, rehit, result, att, rng, status,
                                                            next_tmin);
        if (out == BOUNCE_REHIT) {   // the same depth again
            rehit = true;
            tmin = next_tmin;
            ++depth;
            continue;
        }
        if (out != BOUNCE_NEXT) break;
        rehit = false;
        tmin = 0.00001f;
    }
}

// One camera sample: camera::ray_color (camera.cuh:149-264).  Returns the radiance of the sample.
template <bool CLEAN, int ORDER, class R>
__device__ __forceinline__ RGB trace_sample(const DevScene& S, Ray r, int max_depth, R& rng, PathCounters& pc,
                                            uint32_t& status) {
    RGB result = rgb(0.f, 0.f, 0.f);
    RGB att = rgb(1.f, 1.f, 1.f);
    TraceStats st{0, 0};
    trace_bounces<CLEAN, ORDER>(S, r, max_depth, max_depth, 0.00001f, result, att, rng, pc, st, status);
    pc.nodes += st.nodes;
    pc.prims += st.prims;
    return result;
}

}  // namespace RTC_XP_NS
}  // namespace rtc
