// rtc_wavefront.cuh - wavefront form of the path loop: init / extend / shade kernels over compacted
// slot queues.
//
// A slot holds one pixel in flight.  Its samples run in order on the slot (the compat stream is one
// thrust::minstd_rand per pixel, consumed by all samples, core/src/gpu.cu:770-790), so the radiance
// is bit-identical to the megakernel's.  What changes is the shape of the work:
//   extend  every queued slot runs only the closest-hit traversal of its current ray;
//   shade   every queued slot runs one bounce of camera::ray_color (shade_bounce_deferred); a finished sample
//           adds into the pixel sum and the slot regenerates the next camera sample, a finished pixel
//           is written out and the slot fetches the next pixel from a global counter;
// and survivors are compacted into the next queue with one atomic per warp (ballot + popc + shfl).
// Queue counters live on the device; the host launches batches of iterations and polls the count.
//
// Where a slot's pixels come from is a policy type J:
//   WfOne    one image; scene, parameters and output in kernel parameter space (the plain render);
//   WfTable  a ring of job records (DevJob) in device memory and one global pixel sequence over all
//            admitted jobs (batched and served renders): images of different scenes, cameras,
//            resolutions, spp and depths share the slots, each pixel still computed exactly as the
//            plain render computes it.
#pragma once

#include <type_traits>

// Launch bounds of the iteration kernels (extend, shade, fused bounce), which run with 128, 256 or 512
// threads per block (WfLaunch::block, a batch autotuner knob).  Build-time knobs for occupancy sweeps:
// RTC_EXTEND_MINB / RTC_SHADE_MINB ask for that many resident 512-thread blocks per SM (a register cap of
// 65536 / (512 x blocks)), RTC_EXTEND_MAXNREG caps the extend kernel at any count.  Without them the
// compiler's own choice stands (extend 64 registers); note that an explicit minimum of 1 is not the same
// as none.  The shade kernels are capped at 64 registers (RTC_SHADE_ONE_MAXNREG for a single image,
// RTC_SHADE_MAXNREG for the ring; see wf_shade).
#define RTC_ITER_BLOCK_MAX 512
#if defined(RTC_EXTEND_MAXNREG)
#define RTC_EXTEND_BOUNDS __maxnreg__(RTC_EXTEND_MAXNREG)
#elif defined(RTC_EXTEND_MINB)
#define RTC_EXTEND_BOUNDS __launch_bounds__(RTC_ITER_BLOCK_MAX, RTC_EXTEND_MINB)
#else
#define RTC_EXTEND_BOUNDS __launch_bounds__(RTC_ITER_BLOCK_MAX)
#endif
#if defined(RTC_SHADE_MINB)
#define RTC_SHADE_BOUNDS __launch_bounds__(RTC_ITER_BLOCK_MAX, RTC_SHADE_MINB)
#else
// a register cap (__maxnreg__ cannot be combined with launch bounds); see wf_shade_ring
#ifndef RTC_SHADE_MAXNREG
#define RTC_SHADE_MAXNREG 64
#endif
#define RTC_SHADE_BOUNDS __maxnreg__(RTC_SHADE_MAXNREG)
#endif
#ifdef RTC_FINISH_MINB
#define RTC_FINISH_BOUNDS __launch_bounds__(128, RTC_FINISH_MINB)
#else
#define RTC_FINISH_BOUNDS __launch_bounds__(128)
#endif

#include "rtc_kernels.h"
#include "rtc_path.cuh"

namespace rtc {
inline namespace RTC_XP_NS {

// Loads of the path state (queue entries and slot records): a build-time choice of cache policy - 0
// streaming (ld.global.cs, evict first), 1 L2 only (ld.global.cg: the default), 2 the default policy
// (L1 and L2).  Each slot's state is read once per iteration, so caching it in L1 only evicts node
// records; on the spheres frame (1280x720, 64 spp) 1 measured 2.5% faster than 0 and 0.5% faster
// than 2 (shade 26.0 ms against 27.4 and 26.3 ms).
#ifndef RTC_STATE_LOAD
#define RTC_STATE_LOAD 1
#endif
template <class T>
__device__ __forceinline__ T ld_state(const T* p) {
#if RTC_STATE_LOAD == 1
    return __ldcg(p);
#elif RTC_STATE_LOAD == 2
    return *p;
#else
    return __ldcs(p);
#endif
}

// ---- slot records (WfBuffers::rec): three 32-byte sectors per slot, one 256-bit access each --------

struct Sec {
    uint32_t w[8];
};
constexpr int SEC_RAY = 0, SEC_SHADE = 1, SEC_PIXEL = 2;

__device__ __forceinline__ uint32_t* wf_sec(const WfBuffers& B, uint32_t slot, int sec) {
    return B.rec + (size_t)slot * WF_REC_WORDS + 8 * sec;
}

__device__ __forceinline__ Sec ld_sec(const uint32_t* p) {
    Sec s;
#if RTC_STATE_LOAD == 1
    asm volatile("ld.global.cg.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
#elif RTC_STATE_LOAD == 2
    asm volatile("ld.global.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
#else
    asm volatile("ld.global.cs.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
#endif
                 : "=r"(s.w[0]), "=r"(s.w[1]), "=r"(s.w[2]), "=r"(s.w[3]), "=r"(s.w[4]), "=r"(s.w[5]), "=r"(s.w[6]),
                   "=r"(s.w[7])
                 : "l"(p));
    return s;
}

// A record load is a volatile asm without a memory clobber, and every store into the records is a
// volatile asm with one: the loads keep their order against the stores (no volatile asm passes
// another) without stopping the compiler from keeping scene data in registers across a load.
__device__ __forceinline__ void st_word(uint32_t* p, uint32_t v) {
    asm volatile("st.global.b32 [%0], %1;" : : "l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_word(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.cg.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ void st_sec(uint32_t* p, const Sec& s) {
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
                 :
                 : "l"(p), "r"(s.w[0]), "r"(s.w[1]), "r"(s.w[2]), "r"(s.w[3]), "r"(s.w[4]), "r"(s.w[5]), "r"(s.w[6]),
                   "r"(s.w[7])
                 : "memory");
}

// sector 0: origin, direction, the trace's start, the depth word
__device__ __forceinline__ Sec ray_sec(V3 o, V3 d, float start, uint32_t mw) {
    Sec s;
    s.w[0] = __float_as_uint(o.x);
    s.w[1] = __float_as_uint(o.y);
    s.w[2] = __float_as_uint(o.z);
    s.w[3] = __float_as_uint(d.x);
    s.w[4] = __float_as_uint(d.y);
    s.w[5] = __float_as_uint(d.z);
    s.w[6] = __float_as_uint(start);
    s.w[7] = mw;
    return s;
}
__device__ __forceinline__ V3 sec_v3(const Sec& s, int k) {
    return v3(__uint_as_float(s.w[k]), __uint_as_float(s.w[k + 1]), __uint_as_float(s.w[k + 2]));
}
__device__ __forceinline__ float sec_f(const Sec& s, int k) { return __uint_as_float(s.w[k]); }

// sector 1: attenuation, sample radiance (the hit words are the extend kernel's to write)
__device__ __forceinline__ Sec shade_sec(RGB att, RGB acc) {
    Sec s;
    s.w[0] = __float_as_uint(att.r);
    s.w[1] = __float_as_uint(att.g);
    s.w[2] = __float_as_uint(att.b);
    s.w[3] = __float_as_uint(acc.r);
    s.w[4] = __float_as_uint(acc.g);
    s.w[5] = __float_as_uint(acc.b);
    s.w[6] = 0u;
    s.w[7] = 0xffffffffu;
    return s;
}

// the closest hit (t, item bits) into sector 1's last two words
__device__ __forceinline__ void st_hit(uint32_t* shade_sector, float t, uint32_t item) {
    asm volatile("st.global.v2.b32 [%0], {%1, %2};" : : "l"(shade_sector + 6), "r"(__float_as_uint(t)), "r"(item)
                 : "memory");
}

// sector 2: pixel, sample, minstd state / sample group, PCG32 state, pixel sum
__device__ __forceinline__ Sec pixel_sec(uint32_t pixel, uint32_t sample, uint32_t aux, uint64_t pcg_state, float4 ps) {
    Sec s;
    s.w[0] = pixel;
    s.w[1] = sample;
    s.w[2] = aux;
    s.w[3] = (uint32_t)pcg_state;
    s.w[4] = __float_as_uint(ps.x);
    s.w[5] = __float_as_uint(ps.y);
    s.w[6] = __float_as_uint(ps.z);
    s.w[7] = (uint32_t)(pcg_state >> 32);
    return s;
}
__device__ __forceinline__ float4 sec_psum(const Sec& s) {
    return make_float4(__uint_as_float(s.w[4]), __uint_as_float(s.w[5]), __uint_as_float(s.w[6]), 0.0f);
}

// A slot's ray sector carries the start of its trace: 0 for an ordinary ray (tmin = 1e-5,
// SHADOW_ACNE_FIX, constants.cuh:27), or t + 0.001 for the re-hit from behind a one-sided light that
// the shade kernel hands back to the extend kernel (camera.cuh:177-183).
__device__ __forceinline__ float wf_tmin(float start) { return start > 0.0f ? start : 0.00001f; }

// Work distribution of the iteration kernels, in chunks of 32 queue entries per warp:
//   fixed    warp w of the grid takes chunks w, w + W, w + 2W, ... (W warps in the grid);
//   dynamic  a warp takes the next chunk from a counter (one atomic by lane 0), and asks for its
//            following chunk before it works on the current one, so the atomic's round trip overlaps
//            the work.
// Dynamic pays where walks are long and uneven (triangle meshes, a batch of many scenes): with the
// fixed stride the warps that drew long walks ran alone at the end of each launch.  Where walks are
// short (the 489-primitive spheres frame), the atomics on one counter cost more than the imbalance.
// The choice is a template parameter, so the fixed form compiles to the plain grid-stride loop.  Every
// lane of the warp must call it together.
template <bool DYN>
struct WfChunks {
    uint32_t* ctr;
    uint32_t next;
    __device__ __forceinline__ explicit WfChunks(uint32_t* c) : ctr(c) {
        uint32_t b = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
        if constexpr (DYN) {
            if ((threadIdx.x & 31) == 0) b = atomicAdd(ctr, 32u);
            b = __shfl_sync(0xffffffffu, b, 0);
        }
        next = b;
    }
    // the current chunk's first entry, and the request for the one after it
    __device__ __forceinline__ uint32_t take(uint32_t& pending) {
        const uint32_t base = next;
        pending = 0;
        if constexpr (DYN) {
            if ((threadIdx.x & 31) == 0) pending = atomicAdd(ctr, 32u);
        }
        return base;
    }
    __device__ __forceinline__ void advance(uint32_t pending) {
        if constexpr (DYN) next = __shfl_sync(0xffffffffu, pending, 0);
        else next += gridDim.x * blockDim.x;
    }
};

// Appends `slot` to queue `q` when `pred`; every active lane of the warp must call it together.
__device__ __forceinline__ void wf_push(uint32_t* q, uint32_t* cnt, uint32_t slot, bool pred) {
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, pred);
    if (m == 0u) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(cnt, (uint32_t)__popc(m));
    base = __shfl_sync(act, base, leader);
    if (pred) q[base + (uint32_t)__popc(m & ((1u << lane) - 1u))] = slot;
}

template <bool CLEAN>
struct WfRngT {
    using type = Minstd;
};
template <>
struct WfRngT<true> {
    using type = Pcg32;
};
template <bool CLEAN>
using WfRng = typename WfRngT<CLEAN>::type;

// The stream of a slot from its pixel sector: compat keeps the minstd state in word 2; clean keeps the
// PCG32 state in words 3 and 7, and the increment of sample s's stream is 2 s + 1 (Pcg32::seed).
template <bool CLEAN>
__device__ __forceinline__ void rng_load(const Sec& px, WfRng<CLEAN>& r) {
    if constexpr (CLEAN) {
        r.state = ((uint64_t)px.w[7] << 32) | px.w[3];
        r.inc = ((uint64_t)px.w[1] << 1) | 1u;
    } else {
        r.x = px.w[2];
    }
}



// Starts sample `s` of pixel `pixel`: jitter and camera ray (perspective_camera::get_ray).
// Compat: one shared stream per pixel, samples in stratum order (gpu.cu:776-786).
// Clean: a PCG32 stream per (pixel, sample).
template <bool CLEAN, int ORDER>
__device__ __forceinline__ void wf_start_sample(const DevScene& S, const DevParams& P, WfRng<CLEAN>& rng,
                                                uint32_t pixel, uint32_t s, Ray& r) {
    const int i = (int)(pixel % (uint32_t)P.width);
    const int j = (int)(pixel / (uint32_t)P.width);
    if constexpr (CLEAN) {
        rng.seed(mix64(((uint64_t)P.seed << 32) ^ (uint64_t)pixel), (uint64_t)s);
        float ju = rng.uniform(), jv = rng.uniform();
        float u = ((float)i + ju) / (float)P.width;
        float v = ((float)j + jv) / (float)P.height;
        r = camera_ray<0>(S.cam, u, v, rng);
    } else {
        const int sq = P.sqrt_spp;
        const int s_j = (int)s / sq, s_i = (int)s % sq;
        float ur = rng.uniform();
        float u = ((float)i + ((float)s_i + ur) / (float)sq) / (float)P.width;
        float v = ((float)j + ((float)s_j + ur) / (float)sq) / (float)P.height;
        r = camera_ray<ORDER>(S.cam, u, v, rng);
    }
}

// The pixel sector's stream words after `rng` has advanced (compat: word 2; clean: words 3 and 7).
template <bool CLEAN>
__device__ __forceinline__ void rng_store(Sec& px, const WfRng<CLEAN>& rng) {
    if constexpr (CLEAN) {
        px.w[3] = (uint32_t)rng.state;
        px.w[7] = (uint32_t)(rng.state >> 32);
    } else {
        px.w[2] = rng.x;
    }
}

__device__ __forceinline__ uint32_t wf_samples(const DevParams& P, bool clean) {
    return clean ? (uint32_t)P.spp : (uint32_t)(P.sqrt_spp * P.sqrt_spp);
}

// Sample groups (clean mode with RTC_FLAG_SAMPLE_GROUPS): a pixel's samples are split into P.groups
// consecutive ranges, each its own work unit on its own slot; group g covers samples
// [g*spp/G, (g+1)*spp/G).  Compat mode always has one group (its samples share one stream).
__device__ __forceinline__ uint32_t wf_group_begin(const DevParams& P, uint32_t g) {
    return (uint32_t)(((uint64_t)g * (uint64_t)P.spp) / (uint64_t)P.groups);
}
__device__ __forceinline__ uint32_t wf_group_end(const DevParams& P, uint32_t g, bool clean) {
    return g + 1u >= (uint32_t)P.groups ? wf_samples(P, clean) : wf_group_begin(P, g + 1u);
}

// ---- job sources ---------------------------------------------------------------------------------

// One image.  Pixels are handed out by a plain atomicAdd on ctr[WF_NEXT_PIXEL] (overshoot is harmless:
// nothing is admitted later).
struct WfOne : WfOneArgs {
    __device__ __forceinline__ WfWindow window() const { return WfWindow{0ull, 0u, 0u}; }
    __device__ __forceinline__ const DevScene& scene(uint32_t) const { return S; }
    __device__ __forceinline__ const DevParams& params(uint32_t) const { return P; }
    __device__ __forceinline__ float4* output(uint32_t) const { return out; }
    __device__ __forceinline__ float4* partials(uint32_t) const { return part; }
    __device__ __forceinline__ uint32_t* group_counts(uint32_t) const { return gcnt; }
    __device__ __forceinline__ void pixel_done(uint32_t) const {}
    // claims the next work unit (pixel x sample group)
    __device__ __forceinline__ bool claim(const WfBuffers& B, const WfWindow&, uint32_t& job, uint32_t& unit,
                                          uint32_t&) const {
        const uint32_t p = atomicAdd(B.ctr + WF_NEXT_PIXEL, 1u);
        if ((int64_t)p >= P.num_pixels * (int64_t)P.groups) return false;
        job = 0u;
        unit = p;
        return true;
    }
};

// A ring of jobs.  The lanes of a warp that need a pixel claim consecutive indices of the global pixel
// sequence with one atomicAdd by the warp's leader; indices at or past the admitted limit are refused
// (the cursor may run past the limit, and the next admission moves it back to the old limit before it
// extends the sequence, so no pixel is skipped).  The owning job is found by binary search over the
// ring's first-pixel indices.
struct WfTable : WfTableArgs {
    __device__ __forceinline__ WfWindow window() const {
        const volatile WfFeed* f = feed;
        WfWindow w;
        w.limit = f->win.limit;
        w.lo = f->win.lo;
        w.hi = f->win.hi;
        return w;
    }
    __device__ __forceinline__ const DevScene& scene(uint32_t j) const { return jobs[j].S; }
    __device__ __forceinline__ const DevParams& params(uint32_t j) const { return jobs[j].P; }
    __device__ __forceinline__ float4* output(uint32_t j) const { return jobs[j].out; }
    __device__ __forceinline__ float4* partials(uint32_t j) const { return jobs[j].part; }
    __device__ __forceinline__ uint32_t* group_counts(uint32_t j) const { return jobs[j].gcnt; }
    __device__ __forceinline__ void pixel_done(uint32_t j) const { atomicAdd(done + j, 1u); }
    // claims the next work unit (pixel x sample group) of the global sequence
    __device__ __forceinline__ bool claim(const WfBuffers&, const WfWindow& win, uint32_t& job, uint32_t& unit,
                                          uint32_t&) const {
        const unsigned act = __activemask();
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(act) - 1;
        unsigned long long base = 0ull;
        if (lane == leader) base = atomicAdd(&feed->next, (unsigned long long)__popc(act));
        base = __shfl_sync(act, base, leader);
        const unsigned long long g = base + (unsigned long long)__popc(act & ((1u << lane) - 1u));
        if (g >= win.limit) return false;
        uint32_t lo = win.lo, hi = win.hi;   // jobs[lo].begin <= g < jobs[hi].begin (hi exclusive)
        while (hi - lo > 1u) {
            const uint32_t mid = lo + (hi - lo) / 2u;
            if (jobs[mid & mask].begin <= g) lo = mid;
            else hi = mid;
        }
        job = lo & mask;
        unit = (uint32_t)(g - jobs[job].begin);
        return true;
    }
};

// Fetches the next pixel for a slot and starts its first sample; returns false when none is left.
template <bool CLEAN, int ORDER, class J>
__device__ __forceinline__ bool wf_fetch_pixel(const J& jobs, const WfWindow& win, const WfBuffers& B, uint32_t slot,
                                               uint32_t& status) {
    uint32_t job = 0, unit = 0;
    if (!jobs.claim(B, win, job, unit, status)) {
        st_word(wf_sec(B, slot, SEC_PIXEL), WF_IDLE);
        return false;
    }
    const DevScene& S = jobs.scene(job);
    const DevParams& P = jobs.params(job);
    const uint32_t G = (uint32_t)P.groups;
    const uint32_t pixel = G > 1u ? unit / G : unit, grp = G > 1u ? unit % G : 0u;
    const uint32_t s0 = G > 1u ? wf_group_begin(P, grp) : 0u;
    WfRng<CLEAN> rng;
    if constexpr (!CLEAN) rng.seed(P.seed + pixel);
    Ray r;
    wf_start_sample<CLEAN, ORDER>(S, P, rng, pixel, s0, r);
    st_sec(wf_sec(B, slot, SEC_RAY), ray_sec(r.o, r.d, 0.0f, wf_pack((uint32_t)P.max_depth, job)));
    st_sec(wf_sec(B, slot, SEC_SHADE), shade_sec(rgb(1.f, 1.f, 1.f), rgb(0.f, 0.f, 0.f)));
    Sec px = pixel_sec(pixel, s0, grp, 0ull, make_float4(0.f, 0.f, 0.f, 0.f));   // clean: word 2 = group
    rng_store<CLEAN>(px, rng);
    st_sec(wf_sec(B, slot, SEC_PIXEL), px);
    return true;
}

// A finished sample group: with one group the pixel's sum is final; otherwise the group's sum is
// stored, and the last group of the pixel to finish adds the partial sums in group order (so the
// result does not depend on which group finished last).
template <class J>
__device__ __forceinline__ void wf_group_done(const J& jobs, uint32_t job, uint32_t pixel, uint32_t grp, float4 ps) {
    const DevParams& P = jobs.params(job);
    if (P.groups <= 1) {
        jobs.output(job)[pixel] = make_float4(ps.x, ps.y, ps.z, 1.0f);
        if (P.rgb8) quantize_pixel(make_float4(ps.x, ps.y, ps.z, 1.0f), P.spp, P.width, P.height, pixel, P.rgb8);
        jobs.pixel_done(job);
        return;
    }
    float4* part = jobs.partials(job) + (size_t)pixel * (size_t)P.groups;
    part[grp] = ps;
    __threadfence();
    if (atomicAdd(jobs.group_counts(job) + pixel, 1u) != (uint32_t)P.groups - 1u) return;
    __threadfence();
    float4 t = __ldcg(part);
    for (int g = 1; g < P.groups; ++g) {
        const float4 v = __ldcg(part + g);
        t.x += v.x;
        t.y += v.y;
        t.z += v.z;
    }
    jobs.output(job)[pixel] = make_float4(t.x, t.y, t.z, 1.0f);
    if (P.rgb8) quantize_pixel(make_float4(t.x, t.y, t.z, 1.0f), P.spp, P.width, P.height, pixel, P.rgb8);
    jobs.pixel_done(job);
}

// First fill of a single-image render: slot k takes a pixel, joins queue 0.
template <bool CLEAN, int ORDER>
__global__ void __launch_bounds__(128) wf_init(WfOne J, WfBuffers B) {
    uint32_t status = 0;
    const WfWindow win = J.window();
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < B.slots; base += stride) {
        const uint32_t slot = base + threadIdx.x;
        bool live = false;
        if (slot < B.slots) live = wf_fetch_pixel<CLEAN, ORDER>(J, win, B, slot, status);
        wf_push(B.queue[0], B.ctr + 0, slot, live);
    }
}

// Publishes a new window of the job ring (one thread, in stream order between iterations): the claim
// cursor moves back to the previous limit if refused claims ran past it, then the window widens.
static __global__ void wf_feed_set(WfFeed* f, WfWindow win) {
    const unsigned long long old = f->win.limit;
    if (f->next > old) f->next = old;
    f->win = win;
}

// Admission: every idle slot claims a pixel of the admitted jobs and joins the queue iteration `w`
// reads.  Runs in stream order between iterations, after wf_feed_set.
template <bool CLEAN, int ORDER>
__global__ void __launch_bounds__(128) wf_admit(WfTable J, WfBuffers B, WfIter w, WfWindow win, uint32_t* status_word) {
    uint32_t status = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < B.slots; base += stride) {
        const uint32_t slot = base + threadIdx.x;
        bool live = false;
        if (slot < B.slots && ld_word(wf_sec(B, slot, SEC_PIXEL)) == WF_IDLE) live = wf_fetch_pixel<CLEAN, ORDER>(J, win, B, slot, status);
        wf_push(B.queue[w.qin], B.ctr + w.cin, slot, live);
    }
    if (status) atomicOr(status_word, status);
}

// FLAVOR: 0 nvcc flavour, 1 g++ flavour, 2 clean mode (double-precision sphere test).
// WIDE: the 8-wide node layout (RTC_FLAG_WIDE_BVH; the other kernels always walk the binary nodes).
template <bool COUNT, int FLAVOR, class J, bool WIDE, bool DYN>
__global__ void RTC_EXTEND_BOUNDS wf_extend(J jobs, WfBuffers B, WfIter w, unsigned long long* counters,
                                                 uint32_t* status_word) {
    const uint32_t n = B.ctr[w.cin];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        B.ctr[w.czero] = 0u;
        B.ctr[WF_FETCH_SHADE] = 0u;   // the shade kernel that follows hands out its entries from 0
    }
    const uint32_t* q = B.queue[w.qin];
    TraceStats st{0, 0};
    uint32_t status = 0, rays = 0;
    WfChunks<DYN> chunks(B.ctr + WF_FETCH_EXTEND);
    for (;;) {
        uint32_t pending;
        const uint32_t base = chunks.take(pending);
        if (base >= n) break;   // the same for the whole warp
        const uint32_t k = base + (threadIdx.x & 31u);
        if (k < n) {
            const uint32_t slot = ld_state(q + k);
            const Sec R = ld_sec(wf_sec(B, slot, SEC_RAY));
            const uint32_t mw = R.w[7];
            const uint32_t job = wf_job(mw);
            float t;
            uint32_t item;
            bool h = closest_hit<FLAVOR == 2, WIDE>(jobs.scene(job), sec_v3(R, 0), sec_v3(R, 3), wf_tmin(sec_f(R, 6)),
                                                    3.402823466e+38f,
                                                    wf_depth(mw) == (uint32_t)jobs.params(job).max_depth, t, item, st,
                                                    status);
            st_hit(wf_sec(B, slot, SEC_SHADE), t, h ? item : 0xffffffffu);
            ++rays;
        }
        chunks.advance(pending);   // one call site: every lane of the warp takes part
    }
    if (COUNT && counters) {
        unsigned long long r = rays, nn = st.nodes, pp = st.prims;
        for (int off = 16; off > 0; off >>= 1) {
            r += __shfl_down_sync(0xffffffffu, r, off);
            nn += __shfl_down_sync(0xffffffffu, nn, off);
            pp += __shfl_down_sync(0xffffffffu, pp, off);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(counters + CNT_RAYS, r);
            atomicAdd(counters + CNT_NODES, nn);
            atomicAdd(counters + CNT_PRIMS, pp);
            atomicAdd(counters + CNT_EXT_RAYS, r);
            atomicAdd(counters + CNT_EXT_NODES, nn);
            atomicAdd(counters + CNT_EXT_PRIMS, pp);
        }
    }
    if (status) atomicOr(status_word, status);
}

// One shade step of a slot whose current ray has been traced: shade_bounce_deferred, then the slot's
// bookkeeping (next bounce / next sample / next pixel).  Returns true while the slot has a ray to trace.
template <bool CLEAN, int ORDER, class J>
__device__ __forceinline__ bool wf_step(const J& jobs, const WfWindow& win, const WfBuffers& B, uint32_t slot,
                                        const Sec& R, const Sec& SH, const Sec& PX, float t, uint32_t item,
                                        PathCounters& pc, TraceStats& st, uint32_t& paths, uint32_t& status) {
    const uint32_t job = wf_job(R.w[7]);
    // local copies: a job record in the ring is read once here; through a reference it would be
    // re-read after each store to the path state below, which the compiler cannot prove does not alias
    // it (a single image's record is in kernel parameters either way)
    const DevScene S = jobs.scene(job);
    const DevParams P = jobs.params(job);
    Ray r;
    r.o = sec_v3(R, 0);
    r.d = sec_v3(R, 3);
    r.time = 0.0f;
    RGB att = rgb(sec_f(SH, 0), sec_f(SH, 1), sec_f(SH, 2)), acc = rgb(sec_f(SH, 3), sec_f(SH, 4), sec_f(SH, 5));
    WfRng<CLEAN> rng;
    rng_load<CLEAN>(PX, rng);   // of the pixel sector only the stream is kept past this point
    uint32_t depth = wf_depth(R.w[7]);
    float rehit_tmin = 0.0f;
    const int out = shade_bounce_deferred<CLEAN, ORDER>(S, r, item != 0xffffffffu, t, item, sec_f(R, 6) > 0.0f, acc,
                                                        att, rng, status, rehit_tmin);
    uint32_t* rec_ray = wf_sec(B, slot, SEC_RAY);
    uint32_t* rec_shade = wf_sec(B, slot, SEC_SHADE);
    uint32_t* rec_px = wf_sec(B, slot, SEC_PIXEL);
    if (out == BOUNCE_REHIT) {
        // the same ray again from behind the light, at the same depth: only the radiance and the ray's
        // start change (no random draw has been made)
        st_sec(rec_ray, ray_sec(r.o, r.d, rehit_tmin, R.w[7]));
        st_sec(rec_shade, shade_sec(att, acc));
        return true;
    }
    const bool cont = out == BOUNCE_NEXT;
    if (cont) --depth;
    if (cont && depth > 0u) {
        // the path continues: next bounce (of the pixel sector only the stream words change)
        st_sec(rec_ray, ray_sec(r.o, r.d, 0.0f, wf_pack(depth, job)));
        st_sec(rec_shade, shade_sec(att, acc));
        if constexpr (CLEAN) {
            st_word(rec_px + 3, (uint32_t)rng.state);
            st_word(rec_px + 7, (uint32_t)(rng.state >> 32));
        } else {
            st_word(rec_px + 2, rng.x);
        }
        return true;
    }
    // the sample is done: pixel_color += ray_color(...) (gpu.cu:787).  The pixel sector is read again
    // here (a quarter of the bounces end a sample) rather than held in registers through the bounce.
    ++paths;
    const Sec px = ld_sec(rec_px);
    float4 ps = sec_psum(px);
    if (!CLEAN || (isfinite(acc.r) && isfinite(acc.g) && isfinite(acc.b))) {
        ps.x += acc.r;
        ps.y += acc.g;
        ps.z += acc.b;
    }
    const uint32_t pixel = px.w[0];
    const uint32_t s = px.w[1] + 1u;
    const uint32_t grp = CLEAN ? px.w[2] : 0u;
    if (s < (P.groups > 1 ? wf_group_end(P, grp, CLEAN) : wf_samples(P, CLEAN))) {
        // regenerate: the pixel's next sample on the same slot
        Ray nr;
        wf_start_sample<CLEAN, ORDER>(S, P, rng, pixel, s, nr);
        st_sec(rec_ray, ray_sec(nr.o, nr.d, 0.0f, wf_pack((uint32_t)P.max_depth, job)));
        st_sec(rec_shade, shade_sec(rgb(1.f, 1.f, 1.f), rgb(0.f, 0.f, 0.f)));
        Sec npx = pixel_sec(pixel, s, px.w[2], 0ull, ps);
        rng_store<CLEAN>(npx, rng);
        st_sec(rec_px, npx);
        return true;
    }
    // the pixel (or its sample group) is done: write it and take the next work unit
    wf_group_done(jobs, job, pixel, grp, ps);
    return wf_fetch_pixel<CLEAN, ORDER>(jobs, win, B, slot, status);
}

template <bool COUNT>
__device__ __forceinline__ void wf_flush(unsigned long long* counters, uint32_t rays, uint32_t paths, const TraceStats& st) {
    if (!COUNT || !counters) return;
    unsigned long long r = rays, p = paths, nn = st.nodes, pp = st.prims;
    for (int off = 16; off > 0; off >>= 1) {
        r += __shfl_down_sync(0xffffffffu, r, off);
        p += __shfl_down_sync(0xffffffffu, p, off);
        nn += __shfl_down_sync(0xffffffffu, nn, off);
        pp += __shfl_down_sync(0xffffffffu, pp, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counters + CNT_RAYS, r);
        atomicAdd(counters + CNT_PATHS, p);
        atomicAdd(counters + CNT_NODES, nn);
        atomicAdd(counters + CNT_PRIMS, pp);
    }
}

template <bool CLEAN, int ORDER, bool COUNT, bool DYN, class J>
__device__ __forceinline__ void wf_shade_pass(const J& jobs, const WfBuffers& B, WfIter w, unsigned long long* counters,
                                              uint32_t* status_word) {
    const uint32_t n = B.ctr[w.cin];
    const WfWindow win = jobs.window();
    const uint32_t* q = B.queue[w.qin];
    uint32_t* qn = B.queue[w.qin ^ 1];
    uint32_t* cn = B.ctr + w.cout;
    uint32_t status = 0, paths = 0;
    PathCounters pc{0, 0, 0};
    TraceStats st{0, 0};
    if (blockIdx.x == 0 && threadIdx.x == 0) B.ctr[WF_FETCH_EXTEND] = 0u;   // for the next extend kernel
    WfChunks<DYN> chunks(B.ctr + WF_FETCH_SHADE);
    for (;;) {   // whole warps iterate together, so wf_push sees full warps
        uint32_t pending;
        const uint32_t base = chunks.take(pending);
        if (base >= n) break;   // the same for the whole warp
        const uint32_t k = base + (threadIdx.x & 31u);
        bool live = false;
        uint32_t slot = 0;
        if (k < n) {
            slot = ld_state(q + k);
            const Sec R = ld_sec(wf_sec(B, slot, SEC_RAY));
            const Sec SH = ld_sec(wf_sec(B, slot, SEC_SHADE));
            const Sec PX = ld_sec(wf_sec(B, slot, SEC_PIXEL));
            live = wf_step<CLEAN, ORDER>(jobs, win, B, slot, R, SH, PX, sec_f(SH, 6), SH.w[7], pc, st, paths, status);
        }
        wf_push(qn, cn, slot, live);
        chunks.advance(pending);
    }
    wf_flush<COUNT>(counters, pc.rays, paths, st);
    if (status) atomicOr(status_word, status);
}

// The shade kernels.  A single image's shade step is held to RTC_SHADE_ONE_MAXNREG registers (64 by
// default): 8 blocks of 128 threads per SM, so its grid (8 blocks per SM) runs in one wave at more warps
// than the compiler's own 85 registers allow (5 blocks per SM, and the grid's last 3 blocks per SM ran
// alone afterwards).  It spills 32 bytes; on the spheres frame (1280x720, 64 spp) shade fell from 22.2 to
// 17.9 ms per frame, where 80 and 72 registers (6 and 7 blocks, still two waves) measured 23.1 and
// 22.2 ms.  The ring's shade step (batched and served renders), which copies its job record, takes 128
// registers uncapped and spills 256 bytes at 64, yet 64 measured fastest there too: 64 scenes in compat
// mode 846 -> 870 Mpaths/s, where 80 and 96 registers (164 and 92 bytes of spills, 6 and 5 blocks per
// SM) measured 803 and 814.
#ifndef RTC_SHADE_ONE_MAXNREG
#define RTC_SHADE_ONE_MAXNREG 64
#endif
template <bool CLEAN, int ORDER, bool COUNT, bool DYN>
__global__ void __maxnreg__(RTC_SHADE_ONE_MAXNREG) wf_shade(WfOne jobs, WfBuffers B, WfIter w,
                                                            unsigned long long* counters, uint32_t* status_word) {
    wf_shade_pass<CLEAN, ORDER, COUNT, DYN>(jobs, B, w, counters, status_word);
}
template <bool CLEAN, int ORDER, bool COUNT, bool DYN>
__global__ void RTC_SHADE_BOUNDS wf_shade_ring(WfTable jobs, WfBuffers B, WfIter w, unsigned long long* counters,
                                               uint32_t* status_word) {
    wf_shade_pass<CLEAN, ORDER, COUNT, DYN>(jobs, B, w, counters, status_word);
}

// Fused form of one iteration: trace + shade of every queued slot in one launch (each lane still does
// exactly one bounce, so the warp stays in the same phase), then compaction into the next queue.
template <bool CLEAN, int ORDER, bool COUNT, class J>
__global__ void __launch_bounds__(RTC_ITER_BLOCK_MAX) wf_bounce(J jobs, WfBuffers B, WfIter w, unsigned long long* counters,
                                                 uint32_t* status_word) {
    const uint32_t n = B.ctr[w.cin];
    if (blockIdx.x == 0 && threadIdx.x == 0) B.ctr[w.czero] = 0u;   // appended to by the next iteration
    const WfWindow win = jobs.window();
    const uint32_t* q = B.queue[w.qin];
    uint32_t* qn = B.queue[w.qin ^ 1];
    uint32_t* cn = B.ctr + w.cout;
    uint32_t status = 0, paths = 0, rays = 0;
    PathCounters pc{0, 0, 0};
    TraceStats st{0, 0};
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t limit = (n + 31u) & ~31u;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < limit; k += stride) {
        bool live = false;
        uint32_t slot = 0;
        if (k < n) {
            slot = ld_state(q + k);
            const Sec R = ld_sec(wf_sec(B, slot, SEC_RAY));
            const Sec SH = ld_sec(wf_sec(B, slot, SEC_SHADE));
            const Sec PX = ld_sec(wf_sec(B, slot, SEC_PIXEL));
            const uint32_t mw = R.w[7];
            const uint32_t job = wf_job(mw);
            float t;
            uint32_t item;
            ++rays;
            bool h = closest_hit<CLEAN>(jobs.scene(job), sec_v3(R, 0), sec_v3(R, 3), wf_tmin(sec_f(R, 6)), 3.402823466e+38f,
                                        wf_depth(mw) == (uint32_t)jobs.params(job).max_depth, t, item, st, status);
            live = wf_step<CLEAN, ORDER>(jobs, win, B, slot, R, SH, PX, t, h ? item : 0xffffffffu, pc, st, paths, status);
        }
        wf_push(qn, cn, slot, live);
    }
    wf_flush<COUNT>(counters, rays + pc.rays, paths, st);
    if (status) atomicOr(status_word, status);
}

// Long-chain split (one pass in place of an iteration): a slot whose predicted remaining work - samples
// left times the iterations each of its samples has taken so far (`k0` iterations since the start) -
// exceeds `threshold` iterations moves to the long-chain queue, which the drain kernel finishes in
// registers on a second stream while the bulk iterations go on with the other slots.  In compat mode
// a pixel's samples share one stream and cannot run in parallel, so the few pixels whose samples keep
// bouncing (glass) are the frame's critical path; the split starts their register-resident loop ~k0
// iterations into the frame instead of at its end.
template <bool CLEAN, class J>
__global__ void __launch_bounds__(128) wf_split(J jobs, WfBuffers B, WfIter w, float k0, float threshold) {
    const uint32_t n = B.ctr[w.cin];
    if (blockIdx.x == 0 && threadIdx.x == 0) B.ctr[w.czero] = 0u;   // appended to by the next iteration
    const uint32_t* q = B.queue[w.qin];
    uint32_t* qn = B.queue[w.qin ^ 1];
    uint32_t* cn = B.ctr + w.cout;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t limit = (n + 31u) & ~31u;   // whole warps, for the warp-aggregated appends
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < limit; k += stride) {
        bool keep = false, longc = false;
        uint32_t slot = 0;
        if (k < n) {
            slot = q[k];
            const uint32_t mw = ld_word(wf_sec(B, slot, SEC_RAY) + 7), sample = ld_word(wf_sec(B, slot, SEC_PIXEL) + 1);
            const uint32_t nsamp = wf_samples(jobs.params(wf_job(mw)), CLEAN);
            const float rem = (float)(nsamp - sample - 1u) * (k0 / ((float)sample + 1.0f));
            longc = rem > threshold;
            keep = !longc;
        }
        wf_push(qn, cn, slot, keep);
        wf_push(B.queue[2], B.ctr + WF_LONG, slot, longc);
    }
}

// Drain phase: once the queue is small, each remaining slot is finished in place by one thread
// instead of paying two kernel launches per bounce for a nearly empty queue.  Pixels whose samples
// have long paths (glass) make this tail thousands of bounces long in compat mode, where a pixel's
// samples cannot run in parallel, so the loop keeps the whole path state in registers (the
// megakernel's loop, resumed from the slot) and touches memory only to write the finished pixel.
template <bool CLEAN, int ORDER, bool COUNT, class J>
__global__ void RTC_FINISH_BOUNDS wf_finish(J jobs, WfBuffers B, WfIter w, unsigned long long* counters,
                                                 uint32_t* status_word) {
    const uint32_t n = B.ctr[w.cin];
    const WfWindow win = jobs.window();
    const uint32_t* q = B.queue[w.qin];
    uint32_t status = 0, paths = 0;
    PathCounters pc{0, 0, 0};
    TraceStats st{0, 0};
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const uint32_t slot = ld_state(q + k);
        const Sec R = ld_sec(wf_sec(B, slot, SEC_RAY)), SH = ld_sec(wf_sec(B, slot, SEC_SHADE)),
                  PX = ld_sec(wf_sec(B, slot, SEC_PIXEL));
        Ray r;
        r.o = sec_v3(R, 0);
        r.d = sec_v3(R, 3);
        r.time = 0.0f;
        RGB att = rgb(sec_f(SH, 0), sec_f(SH, 1), sec_f(SH, 2)), acc = rgb(sec_f(SH, 3), sec_f(SH, 4), sec_f(SH, 5));
        const float4 p4 = sec_psum(PX);
        float pr = p4.x, pg = p4.y, pb = p4.z;
        WfRng<CLEAN> rng;
        rng_load<CLEAN>(PX, rng);
        uint32_t pixel = PX.w[0], sample = PX.w[1], job = wf_job(R.w[7]), grp = CLEAN ? PX.w[2] : 0u;
        int depth = (int)wf_depth(R.w[7]);
        float tmin = wf_tmin(sec_f(R, 6));   // the slot may wait for its re-hit from behind a one-sided light
        // one pass of the loop finishes the current sample of the current pixel
        for (;;) {
            const DevScene& S = jobs.scene(job);
            const DevParams& P = jobs.params(job);
            // the rest of the current sample: camera::ray_color's loop from `depth` down
            trace_bounces<CLEAN, ORDER>(S, r, depth, P.max_depth, tmin, acc, att, rng, pc, st, status);
            ++paths;
            if (!CLEAN || (isfinite(acc.r) && isfinite(acc.g) && isfinite(acc.b))) {
                pr += acc.r;
                pg += acc.g;
                pb += acc.b;
            }
            if (++sample < (P.groups > 1 ? wf_group_end(P, grp, CLEAN) : wf_samples(P, CLEAN))) {
                wf_start_sample<CLEAN, ORDER>(S, P, rng, pixel, sample, r);
                att = rgb(1.f, 1.f, 1.f);
                acc = rgb(0.f, 0.f, 0.f);
                depth = P.max_depth;
                tmin = 0.00001f;
                continue;
            }
            wf_group_done(jobs, job, pixel, grp, make_float4(pr, pg, pb, 0.0f));
            // a slot that still has pixels to take (fewer slots than pixels) continues through memory
            if (!wf_fetch_pixel<CLEAN, ORDER>(jobs, win, B, slot, status)) break;
            const Sec R2 = ld_sec(wf_sec(B, slot, SEC_RAY)), PX2 = ld_sec(wf_sec(B, slot, SEC_PIXEL));
            r.o = sec_v3(R2, 0);
            r.d = sec_v3(R2, 3);
            att = rgb(1.f, 1.f, 1.f);
            acc = rgb(0.f, 0.f, 0.f);
            pr = pg = pb = 0.f;
            rng_load<CLEAN>(PX2, rng);
            pixel = PX2.w[0];
            sample = PX2.w[1];
            grp = CLEAN ? PX2.w[2] : 0u;
            job = wf_job(R2.w[7]);
            depth = (int)wf_depth(R2.w[7]);
            tmin = wf_tmin(sec_f(R2, 6));
            if (status) break;
        }
    }
    wf_flush<COUNT>(counters, pc.rays, paths, st);
    if (status) atomicOr(status_word, status);
}

// Compacting drain.  The plain drain above gives each remaining slot one thread for its whole chain,
// so a warp runs as long as its longest chain while its other lanes idle (3.8 of 32 lanes active on
// the spheres frame).  Here the chains advance one bounce per step, and every `every` steps the live
// slots of a block move, through shared memory, to the block's lowest threads: the live chains stay
// packed into full warps, and the warps left without a slot wait at the block barrier without
// issuing.  Each slot computes exactly what the plain drain computes for it (the same bounce, sample
// and pixel code in the same order); only which thread runs it changes.
//
// A block takes the queue entries b, b + G, b + 2G, ... (G blocks), so pixels that sit together in the
// queue - neighbours, with similar chains - spread over all SMs; entries past G x WF_DRAIN_BLOCK are
// taken in further rounds.
constexpr int WF_DRAIN_WORDS = 23;   // a slot's state in the pool (WF_DRAIN_BLOCK: rtc_kernels.h)

template <bool CLEAN>
struct DrainSlot {
    V3 o, d;
    float tmin;            // 1e-5, or t + 0.001 for a pending re-hit from behind a one-sided light
    RGB att, acc;
    float pr, pg, pb;      // the pixel (or sample group) sum so far
    WfRng<CLEAN> rng;
    uint32_t pixel, sample, mw, grp, slot;
};

template <bool CLEAN>
__device__ __forceinline__ void drain_load(const WfBuffers& B, uint32_t slot, DrainSlot<CLEAN>& x) {
    const Sec R = ld_sec(wf_sec(B, slot, SEC_RAY)), SH = ld_sec(wf_sec(B, slot, SEC_SHADE)),
              PX = ld_sec(wf_sec(B, slot, SEC_PIXEL));
    x.o = sec_v3(R, 0);
    x.d = sec_v3(R, 3);
    x.tmin = wf_tmin(sec_f(R, 6));
    x.mw = R.w[7];
    x.att = rgb(sec_f(SH, 0), sec_f(SH, 1), sec_f(SH, 2));
    x.acc = rgb(sec_f(SH, 3), sec_f(SH, 4), sec_f(SH, 5));
    x.pr = sec_f(PX, 4);
    x.pg = sec_f(PX, 5);
    x.pb = sec_f(PX, 6);
    rng_load<CLEAN>(PX, x.rng);
    x.pixel = PX.w[0];
    x.sample = PX.w[1];
    x.grp = CLEAN ? PX.w[2] : 0u;
    x.slot = slot;
}

// the slot's words in (or out of) the block's shared pool, column `i`
template <bool CLEAN>
__device__ __forceinline__ void drain_put(uint32_t (*pool)[WF_DRAIN_BLOCK], int i, const DrainSlot<CLEAN>& x) {
    const float f[16] = {x.o.x, x.o.y, x.o.z, x.d.x, x.d.y, x.d.z, x.tmin, x.att.r, x.att.g, x.att.b,
                         x.acc.r, x.acc.g, x.acc.b, x.pr, x.pg, x.pb};
#pragma unroll
    for (int k = 0; k < 16; ++k) pool[k][i] = __float_as_uint(f[k]);
    pool[16][i] = x.pixel;
    pool[17][i] = x.sample;
    pool[18][i] = x.mw;
    pool[19][i] = x.grp;
    pool[20][i] = x.slot;
    if constexpr (CLEAN) {
        pool[21][i] = (uint32_t)x.rng.state;
        pool[22][i] = (uint32_t)(x.rng.state >> 32);
    } else {
        pool[21][i] = x.rng.x;
    }
}
template <bool CLEAN>
__device__ __forceinline__ void drain_get(uint32_t (*pool)[WF_DRAIN_BLOCK], int i, DrainSlot<CLEAN>& x) {
    float f[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = __uint_as_float(pool[k][i]);
    x.o = v3(f[0], f[1], f[2]);
    x.d = v3(f[3], f[4], f[5]);
    x.tmin = f[6];
    x.att = rgb(f[7], f[8], f[9]);
    x.acc = rgb(f[10], f[11], f[12]);
    x.pr = f[13];
    x.pg = f[14];
    x.pb = f[15];
    x.pixel = pool[16][i];
    x.sample = pool[17][i];
    x.mw = pool[18][i];
    x.grp = pool[19][i];
    x.slot = pool[20][i];
    if constexpr (CLEAN) {
        x.rng.state = ((uint64_t)pool[22][i] << 32) | pool[21][i];
        x.rng.inc = ((uint64_t)x.sample << 1) | 1u;
    } else {
        x.rng.x = pool[21][i];
    }
}

// One step of a slot: one pass of camera::ray_color's loop body (trace, then shade_bounce_deferred),
// then the sample's and the pixel's bookkeeping when the sample ends - trace_bounces and the plain
// drain's loop, one bounce at a time.  Returns false when the slot has no pixel left.
template <bool CLEAN, int ORDER, class J>
__device__ __forceinline__ bool drain_step(const J& jobs, const WfWindow& win, const WfBuffers& B, DrainSlot<CLEAN>& x,
                                           PathCounters& pc, TraceStats& st, uint32_t& paths, uint32_t& status) {
    const uint32_t job = wf_job(x.mw);
    const DevScene& S = jobs.scene(job);
    const DevParams& P = jobs.params(job);
    uint32_t depth = wf_depth(x.mw);
    Ray r;
    r.o = x.o;
    r.d = x.d;
    r.time = 0.0f;
    float t, next_tmin = 0.0f;
    uint32_t item;
    pc.rays++;
    const bool hit = closest_hit<CLEAN>(S, r.o, r.d, x.tmin, 3.402823466e+38f, depth == (uint32_t)P.max_depth, t,
                                        item, st, status);
    const int out = shade_bounce_deferred<CLEAN, ORDER>(S, r, hit, t, item, x.tmin > 0.00001f, x.acc, x.att, x.rng,
                                                        status, next_tmin);
    if (out == BOUNCE_REHIT) {   // the same ray again from behind the light, at the same depth
        x.tmin = next_tmin;
        return true;
    }
    if (out == BOUNCE_NEXT && --depth > 0u) {
        x.o = r.o;
        x.d = r.d;
        x.tmin = 0.00001f;
        x.mw = wf_pack(depth, job);
        return true;
    }
    // the sample is done: pixel_color += ray_color(...) (gpu.cu:787)
    ++paths;
    if (!CLEAN || (isfinite(x.acc.r) && isfinite(x.acc.g) && isfinite(x.acc.b))) {
        x.pr += x.acc.r;
        x.pg += x.acc.g;
        x.pb += x.acc.b;
    }
    if (++x.sample < (P.groups > 1 ? wf_group_end(P, x.grp, CLEAN) : wf_samples(P, CLEAN))) {
        wf_start_sample<CLEAN, ORDER>(S, P, x.rng, x.pixel, x.sample, r);
        x.o = r.o;
        x.d = r.d;
        x.tmin = 0.00001f;
        x.att = rgb(1.f, 1.f, 1.f);
        x.acc = rgb(0.f, 0.f, 0.f);
        x.mw = wf_pack((uint32_t)P.max_depth, job);
        return true;
    }
    wf_group_done(jobs, job, x.pixel, x.grp, make_float4(x.pr, x.pg, x.pb, 0.0f));
    // a slot that still has pixels to take (fewer slots than pixels) continues through memory
    if (!wf_fetch_pixel<CLEAN, ORDER>(jobs, win, B, x.slot, status)) return false;
    drain_load<CLEAN>(B, x.slot, x);
    return status == 0u;
}

template <bool CLEAN, int ORDER, bool COUNT, class J>
__global__ void __launch_bounds__(WF_DRAIN_BLOCK, 2) wf_finish_packed(J jobs, WfBuffers B, WfIter w, int every,
                                                                  unsigned long long* counters, uint32_t* status_word) {
    __shared__ uint32_t pool[WF_DRAIN_WORDS][WF_DRAIN_BLOCK];
    __shared__ int warp_live[WF_DRAIN_BLOCK / 32];
    const uint32_t n = B.ctr[w.cin];
    const WfWindow win = jobs.window();
    const uint32_t* q = B.queue[w.qin];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t G = gridDim.x;
    uint32_t status = 0, paths = 0;
    PathCounters pc{0, 0, 0};
    TraceStats st{0, 0};
    const int steps = every > 0 ? every : 1;
    for (uint32_t round = 0; round < n; round += G * WF_DRAIN_BLOCK) {
        DrainSlot<CLEAN> x;
        const uint32_t k = round + blockIdx.x + G * (uint32_t)tid;
        bool live = k < n;
        if (live) drain_load<CLEAN>(B, ld_state(q + k), x);
        for (;;) {
            for (int s = 0; s < steps; ++s)
                if (live) live = drain_step<CLEAN, ORDER>(jobs, win, B, x, pc, st, paths, status);
            // compaction: the live slots move to threads 0 .. total-1, in thread order
            const unsigned m = __ballot_sync(0xffffffffu, live);
            __syncthreads();   // every thread is done with the pool's previous contents
            if (lane == 0) warp_live[warp] = __popc(m);
            __syncthreads();
            int base = 0, total = 0;
#pragma unroll
            for (int v = 0; v < WF_DRAIN_BLOCK / 32; ++v) {
                const int c = warp_live[v];
                base += v < warp ? c : 0;
                total += c;
            }
            if (total == 0) break;   // the same for every thread of the block
            if (live) drain_put<CLEAN>(pool, base + __popc(m & ((1u << lane) - 1u)), x);
            __syncthreads();
            live = tid < total;
            if (live) drain_get<CLEAN>(pool, tid, x);
        }
    }
    wf_flush<COUNT>(counters, pc.rays, paths, st);
    if (status) atomicOr(status_word, status);
}

// ---- launch dispatch (instantiated once per translation unit / flavour) ---------------------------

template <int FLAVOR, class J, bool DYN>
cudaError_t wf_launch_extend(const J& jobs, const WfBuffers& B, const WfLaunch& L, int blk, bool c) {
    if (L.wide) {
        if (c) wf_extend<true, FLAVOR, J, true, DYN><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, L.counters, L.status);
        else wf_extend<false, FLAVOR, J, true, DYN><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, nullptr, L.status);
    } else {
        if (c) wf_extend<true, FLAVOR, J, false, DYN><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, L.counters, L.status);
        else wf_extend<false, FLAVOR, J, false, DYN><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, nullptr, L.status);
    }
    return cudaGetLastError();
}
template <bool CLEAN, int ORDER, class J, bool DYN>
cudaError_t wf_launch_shade(const J& jobs, const WfBuffers& B, const WfLaunch& L, int blk, bool c) {
    if constexpr (std::is_same<J, WfOne>::value) {
        if (c) wf_shade<CLEAN, ORDER, true, DYN><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, L.counters, L.status);
        else wf_shade<CLEAN, ORDER, false, DYN><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, nullptr, L.status);
    } else {
        if (c) wf_shade_ring<CLEAN, ORDER, true, DYN><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, L.counters, L.status);
        else wf_shade_ring<CLEAN, ORDER, false, DYN><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, nullptr, L.status);
    }
    return cudaGetLastError();
}

template <bool CLEAN, int ORDER, int FLAVOR, class J, class A>
cudaError_t wf_dispatch(WfOp op, const A& args, const WfBuffers& B, const WfLaunch& L) {
    J jobs;
    static_cast<A&>(jobs) = args;
    const bool c = L.counters != nullptr;
    const int blk = L.block > 0 ? L.block : 128;
    if (blk > RTC_ITER_BLOCK_MAX || blk % 32 != 0) return cudaErrorInvalidValue;
    switch (op) {
    case WF_OP_INIT:
        if constexpr (std::is_same<J, WfOne>::value) wf_init<CLEAN, ORDER><<<L.grid, 128, 0, L.st>>>(jobs, B);
        else return cudaErrorInvalidValue;
        break;
    case WF_OP_ADMIT:
        if constexpr (std::is_same<J, WfTable>::value) {
            wf_feed_set<<<1, 1, 0, L.st>>>(jobs.feed, L.win);
            wf_admit<CLEAN, ORDER><<<L.grid, 128, 0, L.st>>>(jobs, B, L.w, L.win, L.status);
        } else {
            return cudaErrorInvalidValue;
        }
        break;
    case WF_OP_EXTEND:
        if (L.dynamic) return wf_launch_extend<FLAVOR, J, true>(jobs, B, L, blk, c);
        return wf_launch_extend<FLAVOR, J, false>(jobs, B, L, blk, c);
    case WF_OP_SHADE:
        if (L.dynamic) return wf_launch_shade<CLEAN, ORDER, J, true>(jobs, B, L, blk, c);
        return wf_launch_shade<CLEAN, ORDER, J, false>(jobs, B, L, blk, c);
    case WF_OP_FINISH:
        if (L.drain_every > 0) {
            if (c) wf_finish_packed<CLEAN, ORDER, true><<<L.grid, WF_DRAIN_BLOCK, 0, L.st>>>(jobs, B, L.w, L.drain_every,
                                                                                          L.counters, L.status);
            else wf_finish_packed<CLEAN, ORDER, false><<<L.grid, WF_DRAIN_BLOCK, 0, L.st>>>(jobs, B, L.w, L.drain_every,
                                                                                            nullptr, L.status);
        } else {
            if (c) wf_finish<CLEAN, ORDER, true><<<L.grid, 128, 0, L.st>>>(jobs, B, L.w, L.counters, L.status);
            else wf_finish<CLEAN, ORDER, false><<<L.grid, 128, 0, L.st>>>(jobs, B, L.w, nullptr, L.status);
        }
        break;
    case WF_OP_SPLIT:
        wf_split<CLEAN><<<L.grid, 128, 0, L.st>>>(jobs, B, L.w, L.k0, L.threshold);
        break;
    case WF_OP_BOUNCE:
        if (c) wf_bounce<CLEAN, ORDER, true><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, L.counters, L.status);
        else wf_bounce<CLEAN, ORDER, false><<<L.grid, blk, 0, L.st>>>(jobs, B, L.w, nullptr, L.status);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace RTC_XP_NS
}  // namespace rtc
