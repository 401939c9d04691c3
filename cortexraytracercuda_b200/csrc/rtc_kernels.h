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
#if defined(RTC_FLAVOR) && RTC_FLAVOR == 0
#define RTC_FLAVOR_FN(name) RTC_FLAVOR_CAT(name, _dev)
#elif defined(RTC_FLAVOR)
#define RTC_FLAVOR_FN(name) RTC_FLAVOR_CAT(name, _host)
#endif

#define RTC_DECLARE_COMPAT(sfx)                                                                                     \
    cudaError_t rtc_launch_render_compat##sfx(const rtc::DevScene& S, const rtc::DevParams& P, float4* out,        \
                                              unsigned long long* counters, uint32_t* status, int block,            \
                                              cudaStream_t st);                                                     \
    cudaError_t rtc_wf_launch_init_compat##sfx(const rtc::DevScene& S, const rtc::DevParams& P,                   \
                                               const rtc::WfBuffers& B, float4* out, int grid, cudaStream_t st);    \
    cudaError_t rtc_wf_launch_extend##sfx(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B, \
                                          rtc::WfIter w, unsigned long long* counters, uint32_t* status, int grid,  \
                                          cudaStream_t st);                                                         \
    cudaError_t rtc_wf_launch_shade_compat##sfx(const rtc::DevScene& S, const rtc::DevParams& P,                  \
                                                const rtc::WfBuffers& B, rtc::WfIter w, float4* out,              \
                                                unsigned long long* counters, uint32_t* status, int grid,         \
                                                cudaStream_t st);                                                   \
    cudaError_t rtc_wf_launch_finish_compat##sfx(const rtc::DevScene& S, const rtc::DevParams& P,                 \
                                                 const rtc::WfBuffers& B, rtc::WfIter w, float4* out,             \
                                                 unsigned long long* counters, uint32_t* status, int grid,        \
                                                 cudaStream_t st);                                                  \
    cudaError_t rtc_wf_launch_bounce_compat##sfx(const rtc::DevScene& S, const rtc::DevParams& P,                 \
                                                 const rtc::WfBuffers& B, rtc::WfIter w, float4* out,             \
                                                 unsigned long long* counters, uint32_t* status, int grid,        \
                                                 cudaStream_t st);

RTC_DECLARE_COMPAT(_dev)
RTC_DECLARE_COMPAT(_host)

cudaError_t rtc_launch_render_clean(const rtc::DevScene& S, const rtc::DevParams& P, float4* out,
                                    unsigned long long* counters, uint32_t* status, int block, cudaStream_t st);
cudaError_t rtc_launch_trace_closest(const rtc::DevScene& S, const float* rays, uint32_t n, int depth,
                                     int max_depth, int32_t* prim, float* t, uint32_t* status, cudaStream_t st);
cudaError_t rtc_launch_quantize(const float4* sum, uint8_t* rgb8, int width, int height, int spp,
                                cudaStream_t st);

// clean-mode wavefront (wavefront_clean.cu); its extend pass is rtc_wf_launch_extend_dev
cudaError_t rtc_wf_launch_init_clean(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B,
                                     float4* out, int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_shade_clean(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B,
                                      rtc::WfIter w, float4* out, unsigned long long* counters, uint32_t* status,
                                      int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_finish_clean(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B,
                                       rtc::WfIter w, float4* out, unsigned long long* counters, uint32_t* status,
                                       int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_bounce_clean(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B,
                                       rtc::WfIter w, float4* out, unsigned long long* counters, uint32_t* status,
                                       int grid, cudaStream_t st);
