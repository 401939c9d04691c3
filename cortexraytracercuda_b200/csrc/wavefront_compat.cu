// wavefront_compat.cu - wavefront kernels in compat mode, compiled once per reference build flavour
// (RTC_FLAVOR=1: g++ flavour, --fmad=false, bit-identical to render_compat.cu's host flavour;
// RTC_FLAVOR=0: nvcc flavour, --fmad=true), for both job sources (one image, job ring).
#include "rtc_kernels.h"
#include "rtc_wavefront.cuh"

#ifndef RTC_FLAVOR
#error "compile with -DRTC_FLAVOR=0 (nvcc flavour) or -DRTC_FLAVOR=1 (g++ flavour)"
#endif

using namespace rtc;

cudaError_t RTC_FLAVOR_FN(rtc_wf_one_compat)(WfOp op, const WfOneArgs& a, const WfBuffers& B, const WfLaunch& L) {
    return wf_dispatch<false, RTC_FLAVOR, RTC_FLAVOR, WfOne>(op, a, B, L);
}

cudaError_t RTC_FLAVOR_FN(rtc_wf_table_compat)(WfOp op, const WfTableArgs& a, const WfBuffers& B, const WfLaunch& L) {
    return wf_dispatch<false, RTC_FLAVOR, RTC_FLAVOR, WfTable>(op, a, B, L);
}
