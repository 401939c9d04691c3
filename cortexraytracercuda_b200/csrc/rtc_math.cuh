// rtc_math.cuh - FP32 vector arithmetic in the exact operation order of the reference's glm usage.
//
// Compat-mode parity depends on evaluating every float expression of the reference in the same order
// with the same rounding (no FMA contraction; the compat translation unit is built with --fmad=false
// and the host side with -ffp-contract=off).  Each helper states the glm/reference expression it
// reproduces:
//   dot(a, b)        glm compute_dot<vec3>: tmp = a*b; tmp.x + tmp.y + tmp.z   (func_geometric.inl:48-55)
//   cross(a, b)      glm compute_cross                                         (func_geometric.inl:68-79)
//   lensq(v)         vector_length_squared: v.x*v.x + v.y*v.y + v.z*v.z        (misc/vector3.cuh:63-66)
//   unit(v)          unit_vector: v / vector3(len, len, len)                   (misc/vector3.cuh:75-78)
//   reflect(I, N)    glm: I - N * dot(N, I) * 2                                (func_geometric.inl:104-110)
//   refract(I,N,e)   glm compute_refract                                       (func_geometric.inl:113-123)
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define RTC_HD __host__ __device__ __forceinline__

namespace rtc {

struct V3 {
    float x, y, z;
};

RTC_HD V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
RTC_HD V3 v3(const float* p) { return v3(p[0], p[1], p[2]); }
RTC_HD V3 v3(float4 a) { return v3(a.x, a.y, a.z); }
RTC_HD V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
RTC_HD V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
RTC_HD V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
RTC_HD V3 mul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }     // vec * scalar
RTC_HD V3 mul(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }     // scalar * vec
RTC_HD V3 mulv(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
RTC_HD V3 divs(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }    // glm vec / scalar
RTC_HD float dot(V3 a, V3 b) {
    float tx = a.x * b.x, ty = a.y * b.y, tz = a.z * b.z;
    return tx + ty + tz;
}
RTC_HD V3 cross(V3 x, V3 y) {
    return v3(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
RTC_HD float lensq(V3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
RTC_HD float len(V3 v) { return sqrtf(lensq(v)); }
RTC_HD V3 unit(V3 v) {
    float l = sqrtf(lensq(v));
    return v3(v.x / l, v.y / l, v.z / l);
}
RTC_HD V3 reflect(V3 I, V3 N) {
    float d = dot(N, I);
    V3 nd = mul(N, d);
    return sub(I, mul(nd, 2.0f));
}
RTC_HD V3 refract(V3 I, V3 N, float eta) {
    float dv = dot(N, I);
    float k = 1.0f - eta * eta * (1.0f - dv * dv);
    if (k >= 0.0f) {
        float s = eta * dv + sqrtf(k);
        return sub(mul(eta, I), mul(s, N));
    }
    return v3(0.0f, 0.0f, 0.0f);
}
// ray::at (misc/ray.cuh:74-77): orig + t * dir
RTC_HD V3 at(V3 o, V3 d, float t) { return add(o, mul(t, d)); }

// Host/device float <-> int bit casts for packing indices into float4 lanes.
RTC_HD float ibits(int32_t i) {
#ifdef __CUDA_ARCH__
    return __int_as_float(i);
#else
    float f; memcpy(&f, &i, 4); return f;
#endif
}
RTC_HD int32_t fbits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_int(f);
#else
    int32_t i; memcpy(&i, &f, 4); return i;
#endif
}

}  // namespace rtc
