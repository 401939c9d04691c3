// rtc_kernels.h - host-side launchers of the sm_100a kernels (defined in render_*.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rtc_dev.h"

cudaError_t rtc_launch_render_compat(const rtc::DevScene& S, const rtc::DevParams& P, float4* out,
                                     unsigned long long* counters, uint32_t* status, int block, cudaStream_t st);
cudaError_t rtc_launch_render_clean(const rtc::DevScene& S, const rtc::DevParams& P, float4* out,
                                    unsigned long long* counters, uint32_t* status, int block, cudaStream_t st);
cudaError_t rtc_launch_trace_closest(const rtc::DevScene& S, const float* rays, uint32_t n, int depth,
                                     int max_depth, int32_t* prim, float* t, uint32_t* status, cudaStream_t st);
cudaError_t rtc_launch_quantize(const float4* sum, uint8_t* rgb8, int width, int height, int spp,
                                cudaStream_t st);

// wavefront engine (wavefront_compat.cu, wavefront_clean.cu)
cudaError_t rtc_wf_launch_init_compat(int order, const rtc::DevScene& S, const rtc::DevParams& P,
                                      const rtc::WfBuffers& B, float4* out, int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_init_clean(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B,
                                     float4* out, int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_extend(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B, rtc::WfIter w,
                                 unsigned long long* counters, uint32_t* status, int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_shade_compat(int order, const rtc::DevScene& S, const rtc::DevParams& P,
                                       const rtc::WfBuffers& B, rtc::WfIter w, float4* out, unsigned long long* counters,
                                       uint32_t* status, int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_shade_clean(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B,
                                      rtc::WfIter w, float4* out, unsigned long long* counters, uint32_t* status, int grid,
                                      cudaStream_t st);
cudaError_t rtc_wf_launch_finish_compat(int order, const rtc::DevScene& S, const rtc::DevParams& P,
                                        const rtc::WfBuffers& B, rtc::WfIter w, float4* out, unsigned long long* counters,
                                        uint32_t* status, int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_finish_clean(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B,
                                       rtc::WfIter w, float4* out, unsigned long long* counters, uint32_t* status, int grid,
                                       cudaStream_t st);
cudaError_t rtc_wf_launch_bounce_compat(int order, const rtc::DevScene& S, const rtc::DevParams& P,
                                        const rtc::WfBuffers& B, rtc::WfIter w, float4* out, unsigned long long* counters,
                                        uint32_t* status, int grid, cudaStream_t st);
cudaError_t rtc_wf_launch_bounce_clean(const rtc::DevScene& S, const rtc::DevParams& P, const rtc::WfBuffers& B,
                                       rtc::WfIter w, float4* out, unsigned long long* counters, uint32_t* status,
                                       int grid, cudaStream_t st);
