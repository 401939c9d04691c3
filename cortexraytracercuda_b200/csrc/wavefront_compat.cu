// wavefront_compat.cu - wavefront kernels in compat mode (built with --fmad=false like
// render_compat.cu, so they are bit-identical to the compat megakernel) and the extend kernel shared
// by both modes.
#include "rtc_kernels.h"
#include "rtc_wavefront.cuh"

using namespace rtc;


cudaError_t rtc_wf_launch_init_compat(int order, const DevScene& S, const DevParams& P, const WfBuffers& B, float4* out,
                                      int grid, cudaStream_t st) {
    if (order == 1) wf_init<false, 1><<<grid, 128, 0, st>>>(S, P, B, out);
    else wf_init<false, 0><<<grid, 128, 0, st>>>(S, P, B, out);
    return cudaGetLastError();
}

cudaError_t rtc_wf_launch_extend(const DevScene& S, const DevParams& P, const WfBuffers& B, WfIter w,
                                 unsigned long long* counters, uint32_t* status, int grid, cudaStream_t st) {
    if (counters) wf_extend<true><<<grid, 128, 0, st>>>(S, P, B, w, counters, status);
    else wf_extend<false><<<grid, 128, 0, st>>>(S, P, B, w, nullptr, status);
    return cudaGetLastError();
}

cudaError_t rtc_wf_launch_shade_compat(int order, const DevScene& S, const DevParams& P, const WfBuffers& B, WfIter w,
                                       float4* out, unsigned long long* counters, uint32_t* status, int grid,
                                       cudaStream_t st) {
    if (counters) {
        if (order == 1) wf_shade<false, 1, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
        else wf_shade<false, 0, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    } else {
        if (order == 1) wf_shade<false, 1, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
        else wf_shade<false, 0, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    }
    return cudaGetLastError();
}

cudaError_t rtc_wf_launch_finish_compat(int order, const DevScene& S, const DevParams& P, const WfBuffers& B, WfIter w,
                                        float4* out, unsigned long long* counters, uint32_t* status, int grid,
                                        cudaStream_t st) {
    if (counters) {
        if (order == 1) wf_finish<false, 1, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
        else wf_finish<false, 0, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    } else {
        if (order == 1) wf_finish<false, 1, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
        else wf_finish<false, 0, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    }
    return cudaGetLastError();
}

cudaError_t rtc_wf_launch_bounce_compat(int order, const DevScene& S, const DevParams& P, const WfBuffers& B, WfIter w,
                                        float4* out, unsigned long long* counters, uint32_t* status, int grid,
                                        cudaStream_t st) {
    if (counters) {
        if (order == 1) wf_bounce<false, 1, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
        else wf_bounce<false, 0, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    } else {
        if (order == 1) wf_bounce<false, 1, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
        else wf_bounce<false, 0, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    }
    return cudaGetLastError();
}
