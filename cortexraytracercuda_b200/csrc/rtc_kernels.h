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
