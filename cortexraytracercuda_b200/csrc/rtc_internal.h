// rtc_internal.h - helpers shared by the C ABI translation units (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/rtc.h"
#include "rtc_dev.h"

// Makes `device` current for the lifetime of the object and gives the calling thread back its own
// current device afterwards: a public entry point works on the device of its context, scene or server
// without changing which device the caller's later CUDA calls go to.
class RtcDeviceScope {
public:
    explicit RtcDeviceScope(int device) {
        if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
        if (prev_ != device) {
            err_ = cudaSetDevice(device);
            changed_ = err_ == cudaSuccess && prev_ >= 0;
        }
    }
    ~RtcDeviceScope() {
        if (changed_) cudaSetDevice(prev_);
    }
    RtcDeviceScope(const RtcDeviceScope&) = delete;
    RtcDeviceScope& operator=(const RtcDeviceScope&) = delete;
    cudaError_t error() const { return err_; }

private:
    int prev_ = -1;
    bool changed_ = false;
    cudaError_t err_ = cudaSuccess;
};

// bytes of wavefront scratch per path slot, and the layout of `slots` slots starting at `base`
size_t rtc_wf_slot_bytes();
size_t rtc_carve_wavefront(void* base, uint32_t slots, rtc::WfBuffers& B);
// records an error message for rtc_last_error_string() and returns `s`
rtc_status rtc_set_error(rtc_status s, const char* msg);
rtc_status rtc_check_render_params(const rtc_render_params* p);
// device-side view of a scene, and the per-launch parameters of a render
const rtc::DevScene& rtc_scene_dev(const rtc_scene* s);
// the device view a render uses: the 8-wide nodes only when the params ask for RTC_FLAG_WIDE_BVH
rtc::DevScene rtc_scene_view(const rtc_scene* s, const rtc_render_params* p);
// drops the environment-map sampling tables from a view unless the render asks for them (clean mode,
// RTC_FLAG_ENV_SAMPLING)
void rtc_view_env_sampling(rtc::DevScene& S, const rtc_render_params* p);
rtc::DevParams rtc_dev_params(const rtc_render_params* p);
// scratch of an image rendered with sample groups (0 without), and its layout at `base`
size_t rtc_group_bytes(const rtc_render_params* p);
// Drain kernel of the wavefront engines (WfLaunch::drain_every): RTC_WF_DRAIN_EVERY when set, else
// `fallback`.
int rtc_drain_every(int fallback);
// Queue distribution of the extend and shade kernels (WfLaunch::dynamic): RTC_WF_DYNAMIC when set, else
// `fallback`.
bool rtc_dynamic_chunks(bool fallback);
void rtc_carve_groups(void* base, const rtc_render_params* p, float4** part, uint32_t** gcnt);
// perspective_camera::initialize; false for a degenerate camera
bool rtc_make_camera(const rtc_camera& c, rtc::DevCamera& out);
int rtc_scene_device(const rtc_scene* s);
// runs the wavefront engine on caller-provided buffers with synchronous queue polling: no device or
// pinned allocations, no events
rtc_status rtc_run_wavefront_sync(const rtc_scene* s, const rtc_render_params* p, const rtc::WfBuffers& B,
                                  uint32_t* d_status, float4* d_out, cudaStream_t st);
