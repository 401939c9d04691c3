// wavefront_clean.cu - wavefront init/shade/finish kernels in clean mode (FMA contraction on); the
// extend pass is the nvcc-flavour one of wavefront_compat.cu.
#include "rtc_kernels.h"
#include "rtc_wavefront.cuh"

using namespace rtc;

cudaError_t rtc_wf_launch_init_clean(const DevScene& S, const DevParams& P, const WfBuffers& B, float4* out, int grid,
                                     cudaStream_t st) {
    wf_init<true, 0><<<grid, 128, 0, st>>>(S, P, B, out);
    return cudaGetLastError();
}

cudaError_t rtc_wf_launch_shade_clean(const DevScene& S, const DevParams& P, const WfBuffers& B, WfIter w, float4* out,
                                      unsigned long long* counters, uint32_t* status, int grid, cudaStream_t st) {
    if (counters) wf_shade<true, 0, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    else wf_shade<true, 0, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    return cudaGetLastError();
}

cudaError_t rtc_wf_launch_finish_clean(const DevScene& S, const DevParams& P, const WfBuffers& B, WfIter w, float4* out,
                                       unsigned long long* counters, uint32_t* status, int grid, cudaStream_t st) {
    if (counters) wf_finish<true, 0, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    else wf_finish<true, 0, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    return cudaGetLastError();
}

cudaError_t rtc_wf_launch_bounce_clean(const DevScene& S, const DevParams& P, const WfBuffers& B, WfIter w, float4* out,
                                       unsigned long long* counters, uint32_t* status, int grid, cudaStream_t st) {
    if (counters) wf_bounce<true, 0, true><<<grid, 128, 0, st>>>(S, P, B, w, out, counters, status);
    else wf_bounce<true, 0, false><<<grid, 128, 0, st>>>(S, P, B, w, out, nullptr, status);
    return cudaGetLastError();
}
