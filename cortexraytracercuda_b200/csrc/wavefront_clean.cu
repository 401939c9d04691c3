// wavefront_clean.cu - wavefront kernels in clean mode (FMA contraction on), for both job sources.
#include "rtc_kernels.h"
#include "rtc_wavefront.cuh"

using namespace rtc;

cudaError_t RTC_XP_FN(rtc_wf_one_clean)(WfOp op, const WfOneArgs& a, const WfBuffers& B, const WfLaunch& L) {
    return wf_dispatch<true, 0, 2, WfOne>(op, a, B, L);
}

cudaError_t RTC_XP_FN(rtc_wf_table_clean)(WfOp op, const WfTableArgs& a, const WfBuffers& B, const WfLaunch& L) {
    return wf_dispatch<true, 0, 2, WfTable>(op, a, B, L);
}
