// render_clean.cu - clean-mode megakernel (counter-based stream per (pixel, sample), FMA allowed).
//
// Same materials, textures and BVH as compat mode; differences: every sample has its own PCG32 stream
// seeded from (seed, pixel, sample), all spp samples are traced (no floor(sqrt(spp))^2), each axis of the
// pixel jitter gets its own draw, and lambertian surfaces use pure cosine sampling when the scene has
// no light to sample.
#include "rtc_kernels.h"
#include "rtc_path.cuh"

namespace rtc {
inline namespace RTC_XP_NS {

__global__ void __launch_bounds__(128) rtc_render_clean(DevScene S, DevParams P, float4* __restrict__ out,
                                                        unsigned long long* counters, uint32_t* status_word) {
    const int64_t pixel_index = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = pixel_index < P.num_pixels;
    PathCounters pc{0, 0, 0};
    uint32_t paths = 0, status = 0;
    if (active) {
        const int i = (int)(pixel_index % P.width);
        const int j = (int)(pixel_index / P.width);
        // sample groups (RTC_FLAG_SAMPLE_GROUPS): each group summed on its own, then the group sums in
        // group order - the wavefront's arithmetic, where the groups run on separate slots
        const int G = P.groups > 1 ? P.groups : 1;
        float tr = 0.f, tg = 0.f, tb = 0.f;
        for (int g = 0; g < G; ++g) {
        const int s0 = (int)(((int64_t)g * P.spp) / G);
        const int s1 = g + 1 == G ? P.spp : (int)(((int64_t)(g + 1) * P.spp) / G);
        float pr = 0.f, pg = 0.f, pb = 0.f;
        for (int s = s0; s < s1; ++s) {
            Pcg32 rng;
            rng.seed(mix64(((uint64_t)P.seed << 32) ^ (uint64_t)pixel_index), (uint64_t)s);
            float ju = rng.uniform(), jv = rng.uniform();
            float u = ((float)i + ju) / (float)P.width;
            float v = ((float)j + jv) / (float)P.height;
            Ray r = camera_ray<0>(S.cam, u, v, rng);
            RGB c = trace_sample<true, 0>(S, r, P.max_depth, rng, pc, status);
            // NaN/Inf samples (degenerate geometry) are dropped instead of poisoning the pixel
            if (isfinite(c.r) && isfinite(c.g) && isfinite(c.b)) { pr += c.r; pg += c.g; pb += c.b; }
            ++paths;
        }
        if (g == 0) {
            tr = pr;
            tg = pg;
            tb = pb;
        } else {
            tr += pr;
            tg += pg;
            tb += pb;
        }
        }
        out[pixel_index] = make_float4(tr, tg, tb, 1.0f);
        if (P.rgb8) quantize_pixel(make_float4(tr, tg, tb, 1.0f), P.spp, P.width, P.height, pixel_index, P.rgb8);
    }
    if (counters) {
        unsigned long long r = pc.rays, p = paths, n = pc.nodes, q = pc.prims;
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
    if (status) atomicOr(status_word, status);
}

}  // namespace RTC_XP_NS
}  // namespace rtc

using namespace rtc;

cudaError_t RTC_XP_FN(rtc_launch_render_clean)(const DevScene& S, const DevParams& P, float4* out, unsigned long long* counters,
                                    uint32_t* status, int block, cudaStream_t st) {
    (void)block;
    const int threads = 128;
    const unsigned grid = (unsigned)((P.num_pixels + threads - 1) / threads);
    rtc_render_clean<<<grid, threads, 0, st>>>(S, P, out, counters, status);
    return cudaGetLastError();
}
