// wavefront_compat.cu - wavefront kernels in compat mode, compiled once per reference build flavour
// (RTC_FLAVOR=1: g++ flavour, --fmad=false, bit-identical to render_compat.cu's host flavour;
// RTC_FLAVOR=0: nvcc flavour, --fmad=true).  The extend kernel of the nvcc flavour also serves clean
// mode.
#include "rtc_kernels.h"
#include "rtc_wavefront.cuh"

#ifndef RTC_FLAVOR
#error "compile with -DRTC_FLAVOR=0 (nvcc flavour) or -DRTC_FLAVOR=1 (g++ flavour)"
#endif

using namespace rtc;

cudaError_t RTC_FLAVOR_FN(rtc_wf_launch_init_compat)(const DevScene& S, const DevParams& P, const WfBuffers& B,
                                                     float4* out, int grid, cudaStream_t st) {
    wf_init<false, RTC_FLAVOR><<<grid, 128, 0, st>>>(S, P, B, out);
    return cudaGetLastError();
}

cudaError_t RTC_FLAVOR_FN(rtc_wf_launch_extend)(const DevScene& S, const DevParams& P, const WfBuffers& B, WfIter w,
                                                unsigned long long* counters, uint32_t* status, int grid,
                                                cudaStream_t st) {
    if (counters) wf_extend<true, RTC_FLAVOR><<<grid, 128, 0, st>>>(S, P, B, w, counters, status);
    else wf_extend<false, RTC_FLAVOR><<<grid, 128, 0, st>>>(S, P, B, w, nullptr, status);
    return cudaGetLastError();
}

cudaError_t RTC_FLAVOR_FN(rtc_wf_launch_shade_compat)(const DevScene& S, const DevParams& P, const WfBuffers& B,
                                                      WfIter w, float4* out, unsigned long long* counters,
                                                      uint32_t* status, int grid, cudaStream_t st) {
    if (counters) wf_shade<false, RTC_FLAVOR, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    else wf_shade<false, RTC_FLAVOR, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    return cudaGetLastError();
}

cudaError_t RTC_FLAVOR_FN(rtc_wf_launch_finish_compat)(const DevScene& S, const DevParams& P, const WfBuffers& B,
                                                       WfIter w, float4* out, unsigned long long* counters,
                                                       uint32_t* status, int grid, cudaStream_t st) {
    if (counters) wf_finish<false, RTC_FLAVOR, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    else wf_finish<false, RTC_FLAVOR, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    return cudaGetLastError();
}

cudaError_t RTC_FLAVOR_FN(rtc_wf_launch_bounce_compat)(const DevScene& S, const DevParams& P, const WfBuffers& B,
                                                       WfIter w, float4* out, unsigned long long* counters,
                                                       uint32_t* status, int grid, cudaStream_t st) {
    if (counters) wf_bounce<false, RTC_FLAVOR, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    else wf_bounce<false, RTC_FLAVOR, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    return cudaGetLastError();
}
