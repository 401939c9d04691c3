// render_compat.cu - compat-mode kernels (reference semantics, per-pixel minstd stream).
//
// Compiled twice, once per reference build flavour (RTC_FLAVOR):
//   RTC_FLAVOR=1 (g++ flavour, --fmad=false): every float expression restated from the reference is
//     evaluated with the roundings of a g++ build of the reference (no FMA contraction, right-to-left
//     multi-draw order), so the only differences left against it are the last-ulp results of
//     cos/sin/acos/atan2;
//   RTC_FLAVOR=0 (nvcc flavour, --fmad=true): left-to-right draws, FMA contraction and CUDA's float
//     trig, like the reference's own device build.  The reference's image depends on contraction (its
//     shadow-acne epsilon, constants.cuh:27, sits at rounding level for scenes of size ~10^2-10^3), so
//     this flavour reproduces the device build's statistics.
// The BVH slab test uses explicit __fmaf_rn in both.
//
// Kernels:
//   rtc_render_compat<ORDER>  one thread per pixel, all samples of the pixel in sequence
//                             (the render kernel, core/src/gpu.cu:761-790), writes the FP32 sum;
//   rtc_trace_closest         closest hit of arbitrary rays (hit-identity tests);
//                             (color.cuh:289-309, gpu.cu:792-799, 2098-2107).
#include "rtc_kernels.h"
#include "rtc_path.cuh"

#ifndef RTC_FLAVOR
#error "compile with -DRTC_FLAVOR=0 (nvcc flavour) or -DRTC_FLAVOR=1 (g++ flavour)"
#endif

namespace rtc {
inline namespace RTC_XP_NS {

__device__ __forceinline__ void flush_counters(unsigned long long* counters, uint32_t rays, uint32_t paths,
                                               uint32_t nodes, uint32_t prims) {
    if (!counters) return;
    unsigned long long r = rays, p = paths, n = nodes, q = prims;
    for (int off = 16; off > 0; off >>= 1) {
        r += __shfl_down_sync(0xffffffffu, r, off);
        p += __shfl_down_sync(0xffffffffu, p, off);
        n += __shfl_down_sync(0xffffffffu, n, off);
        q += __shfl_down_sync(0xffffffffu, q, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counters + CNT_RAYS, r);
        atomicAdd(counters + CNT_PATHS, p);
        atomicAdd(counters + CNT_NODES, n);
        atomicAdd(counters + CNT_PRIMS, q);
    }
}

template <int ORDER>
__global__ void __launch_bounds__(128) rtc_render_compat(DevScene S, DevParams P, float4* __restrict__ out,
                                                         unsigned long long* counters, uint32_t* status_word) {
    const int64_t pixel_index = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = pixel_index < P.num_pixels;
    PathCounters pc{0, 0, 0};
    uint32_t paths = 0, status = 0;
    if (active) {
        const int i = (int)(pixel_index % P.width);
        const int j = (int)(pixel_index / P.width);
        Minstd rng;
        rng.seed(P.seed + (uint32_t)pixel_index);
        const int sq = P.sqrt_spp;
        float pr = 0.f, pg = 0.f, pb = 0.f;
        for (int s_j = 0; s_j < sq; ++s_j) {
            for (int s_i = 0; s_i < sq; ++s_i) {
                float ur = rng.uniform();
                float u = ((float)i + ((float)s_i + ur) / (float)sq) / (float)P.width;
                float v = ((float)j + ((float)s_j + ur) / (float)sq) / (float)P.height;
                Ray r = camera_ray<ORDER>(S.cam, u, v, rng);
                RGB c = trace_sample<false, ORDER>(S, r, P.max_depth, rng, pc, status);
                pr += c.r;
                pg += c.g;
                pb += c.b;
                ++paths;
            }
        }
        out[pixel_index] = make_float4(pr, pg, pb, 1.0f);
        if (P.rgb8) quantize_pixel(make_float4(pr, pg, pb, 1.0f), P.spp, P.width, P.height, pixel_index, P.rgb8);
    }
    flush_counters(counters, pc.rays, paths, pc.nodes, pc.prims);
    if (status) atomicOr(status_word, status);
}

#if RTC_FLAVOR == 1
__device__ __forceinline__ int32_t item_gid(const DevScene& S, uint32_t it) {
    uint32_t kind = it >> ITEM_KIND_SHIFT, idx = it & ITEM_INDEX_MASK;
    switch (kind) {
    case ITEM_XPRIM: return __ldg(S.xprim + idx).w;
    case ITEM_SPHERE: return __ldg(S.sph_aux + idx).y;
    case ITEM_QUAD: return __float_as_int(__ldg(S.quad + 5 * (size_t)idx + 2).w);
    case ITEM_LIGHT: return __float_as_int(__ldg(S.light + 6 * (size_t)idx + 2).w);
    default: return __float_as_int(__ldg(S.tri + 3 * (size_t)idx + 1).w);
    }
}

template <bool WIDE>
__global__ void __launch_bounds__(128) rtc_trace_closest(DevScene S, const float* __restrict__ rays, uint32_t n,
                                                         int depth, int max_depth, int32_t* prim, float* tout,
                                                         uint32_t* status_word) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float* R = rays + 8 * (size_t)k;
    V3 o = v3(R[0], R[1], R[2]), d = v3(R[4], R[5], R[6]);
    float t;
    uint32_t item, status = 0;
    TraceStats st{0, 0};
    bool h = closest_hit<false, WIDE>(S, o, d, R[3], R[7], depth == max_depth, t, item, st, status);
    if (prim) prim[k] = h ? item_gid(S, item) : -1;
    if (tout) tout[k] = h ? t : INFINITY;
    if (status) atomicOr(status_word, status);
}

#endif  // RTC_FLAVOR == 1

}  // namespace RTC_XP_NS
}  // namespace rtc

using namespace rtc;

cudaError_t RTC_FLAVOR_FN(rtc_launch_render_compat)(const DevScene& S, const DevParams& P, float4* out,
                                                   unsigned long long* counters, uint32_t* status, int block,
                                                   cudaStream_t st) {
    (void)block;
    const int threads = 128;
    const unsigned grid = (unsigned)((P.num_pixels + threads - 1) / threads);
    rtc_render_compat<RTC_FLAVOR><<<grid, threads, 0, st>>>(S, P, out, counters, status);
    return cudaGetLastError();
}

#if RTC_FLAVOR == 1

cudaError_t RTC_XP_FN(rtc_launch_trace_closest)(const DevScene& S, const float* rays, uint32_t n, int depth, int max_depth,
                                     int32_t* prim, float* t, uint32_t* status, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const int threads = 128;
    if (S.nodes8)   // the scene view carries the 8-wide nodes only when they were asked for
        rtc_trace_closest<true><<<(n + threads - 1) / threads, threads, 0, st>>>(S, rays, n, depth, max_depth, prim, t, status);
    else
        rtc_trace_closest<false><<<(n + threads - 1) / threads, threads, 0, st>>>(S, rays, n, depth, max_depth, prim, t, status);
    return cudaGetLastError();
}

#endif  // RTC_FLAVOR == 1
