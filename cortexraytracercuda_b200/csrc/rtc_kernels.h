// rtc_kernels.h - host-side launchers of the sm_100a kernels.
//
// Compat-mode launchers exist once per reference build flavour: *_dev (nvcc flavour: left-to-right
// draws, FMA contraction, float trig) and *_host (g++ flavour: right-to-left draws, no contraction,
// double-evaluated trig).  render_compat.cu and wavefront_compat.cu are compiled once per flavour.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rtc_dev.h"

#define RTC_FLAVOR_CAT2(a, b) a##b
#define RTC_FLAVOR_CAT(a, b) RTC_FLAVOR_CAT2(a, b)
#if RTC_XP
#define RTC_XP_FN(name) RTC_FLAVOR_CAT(name, _x)
#else
#define RTC_XP_FN(name) name
#endif
#if defined(RTC_FLAVOR) && RTC_FLAVOR == 0
#define RTC_FLAVOR_FN(name) RTC_XP_FN(RTC_FLAVOR_CAT(name, _dev))
#elif defined(RTC_FLAVOR)
#define RTC_FLAVOR_FN(name) RTC_XP_FN(RTC_FLAVOR_CAT(name, _host))
#endif

namespace rtc {
constexpr int WF_DRAIN_BLOCK = 256;   // threads per block of the compacting drain (wf_finish_packed)

// Wavefront kernel launches.  One dispatcher per (mode, flavour) and job source; `op` picks the kernel.
enum WfOp {
    WF_OP_INIT = 0, WF_OP_ADMIT = 1, WF_OP_EXTEND = 2, WF_OP_SHADE = 3, WF_OP_FINISH = 4, WF_OP_BOUNCE = 5,
    WF_OP_SPLIT = 6
};
struct WfLaunch {
    WfIter w;
    WfWindow win;                    // ADMIT: the window to publish
    float k0, threshold;             // SPLIT: iterations so far, long-chain threshold (iterations)
    bool wide;                       // EXTEND: walk the 8-wide nodes (where the scene carries them)
    unsigned long long* counters;    // NULL: no instrumentation
    uint32_t* status;
    int grid;
    int block;                       // EXTEND / SHADE / BOUNCE: threads per block (0: 128; at most 512)
    bool dynamic;                    // EXTEND / SHADE: warps take chunks of the queue from a counter (WfChunks)
                                     // instead of a fixed grid stride
    int drain_every;                 // FINISH: 0 the plain drain (128-thread blocks, one thread per slot);
                                     // k > 0 the compacting drain (256-thread blocks, live slots repacked
                                     // every k bounce steps)
    cudaStream_t st;
};
using WfOneFn = cudaError_t (*)(WfOp, const WfOneArgs&, const WfBuffers&, const WfLaunch&);
using WfTableFn = cudaError_t (*)(WfOp, const WfTableArgs&, const WfBuffers&, const WfLaunch&);
}  // namespace rtc

#define RTC_DECLARE_COMPAT(sfx)                                                                                     \
    cudaError_t rtc_launch_render_compat##sfx(const rtc::DevScene& S, const rtc::DevParams& P, float4* out,        \
                                              unsigned long long* counters, uint32_t* status, int block,            \
                                              cudaStream_t st);                                                     \
    cudaError_t rtc_wf_one_compat##sfx(rtc::WfOp op, const rtc::WfOneArgs& a, const rtc::WfBuffers& B,            \
                                       const rtc::WfLaunch& L);                                                     \
    cudaError_t rtc_wf_table_compat##sfx(rtc::WfOp op, const rtc::WfTableArgs& a, const rtc::WfBuffers& B,        \
                                         const rtc::WfLaunch& L);

RTC_DECLARE_COMPAT(_dev)
RTC_DECLARE_COMPAT(_host)
// `_x`: the variants built with RTC_XP=1, for scenes with transformed primitives or boxes
RTC_DECLARE_COMPAT(_dev_x)
RTC_DECLARE_COMPAT(_host_x)

// clean mode (render_clean.cu, wavefront_clean.cu) and closest-hit queries (render_compat.cu)
#define RTC_DECLARE_CLEAN(sfx)                                                                                      \
    cudaError_t rtc_launch_render_clean##sfx(const rtc::DevScene& S, const rtc::DevParams& P, float4* out,         \
                                             unsigned long long* counters, uint32_t* status, int block,             \
                                             cudaStream_t st);                                                      \
    cudaError_t rtc_launch_trace_closest##sfx(const rtc::DevScene& S, const float* rays, uint32_t n, int depth,    \
                                              int max_depth, int32_t* prim, float* t, uint32_t* status,            \
                                              cudaStream_t st);                                                     \
    cudaError_t rtc_wf_one_clean##sfx(rtc::WfOp op, const rtc::WfOneArgs& a, const rtc::WfBuffers& B,             \
                                      const rtc::WfLaunch& L);                                                      \
    cudaError_t rtc_wf_table_clean##sfx(rtc::WfOp op, const rtc::WfTableArgs& a, const rtc::WfBuffers& B,         \
                                        const rtc::WfLaunch& L);
RTC_DECLARE_CLEAN()
RTC_DECLARE_CLEAN(_x)
