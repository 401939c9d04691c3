// render_noalloc.cu - the allocation-free render entry point.
//
// Some callers cannot allocate device memory at render time: code that runs under a fixed memory
// budget handed out once at start-up, a host process whose allocator is owned by another framework
// (a pool it must not bypass), or a render issued from a place where a cudaMalloc would synchronise
// the device or fail under a memory cap.  For them rtc_render_noalloc renders with the same
// wavefront kernels as rtc_render_device, but the path state those kernels need (rays, attenuation,
// sample and pixel sums, RNG state, hit records, the two slot queues, the queue counters and the
// kernel status word) lives in one file-scope device array of fixed size instead of context scratch.
//
// Limits and behaviour:
//   * the array is NOALLOC_SCRATCH_BYTES = 64 MiB; every GPU that loads this library holds it until
//     the process exits;
//   * one path slot per pixel, so one call renders at most RTC_NOALLOC_MAX_PIXELS (508,376) pixels
//     and rejects larger images with RTC_ERR_INVALID_ARGUMENT before touching the GPU;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress, once per
//     device, with that device current); make that first call before any stream capture;
//   * every call shares the array: the counters and the status word are cleared at the start of each
//     call, the rest is fully rewritten; calls that overlap on the GPU (two streams, two threads)
//     race on it;
//   * the call returns when the frame is complete: it polls the queue counter with synchronous
//     copies into a host variable (no pinned memory, no events); a call that fails part-way waits
//     for its queued kernels before it returns;
//   * it always runs the wavefront kernels, untimed: params->engine and RTC_FLAG_KERNEL_TIMING are
//     ignored;
//   * the caller's current device is the same after the call as before it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "rtc_internal.h"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(64) << 20;
constexpr size_t NOALLOC_HEADER_BYTES = 256;   // kernel status word
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_rtc_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
void* g_scratch[MAX_DEVICES] = {};

// Device address of the static array on `device` (current): looked up once per device.
rtc_status scratch_address(int device, void** out) {
    if (device < 0 || device >= MAX_DEVICES) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_rtc_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return rtc_set_error(RTC_ERR_CUDA, (std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e)).c_str());
        g_scratch[device] = p;
    }
    *out = g_scratch[device];
    return RTC_OK;
}

}  // namespace

extern "C" rtc_status rtc_render_noalloc(const rtc_scene* scene, const rtc_render_params* params,
                                         float* d_radiance_sum, void* stream) {
    if (!scene || !params || !d_radiance_sum) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)d_radiance_sum & 15u) != 0)
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "radiance buffer must be 16-byte aligned");
    rtc_status r = rtc_check_render_params(params);
    if (r != RTC_OK) return r;
    if (rtc_group_bytes(params) != 0)
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "RTC_FLAG_SAMPLE_GROUPS needs scratch memory; use rtc_render_device");
    const uint64_t npix = (uint64_t)params->width * (uint64_t)params->height;
    const uint64_t cap = RTC_NOALLOC_MAX_PIXELS;
    if (npix > cap) {
        std::string m = "image has " + std::to_string(npix) + " pixels; the allocation-free render holds at most " +
                        std::to_string(cap) + " (one path slot per pixel in a 64 MiB static array)";
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, m.c_str());
    }
    const int device = rtc_scene_device(scene);
    RtcDeviceScope dev(device);   // the caller's current device is restored on return
    cudaError_t e = dev.error();
    if (e != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, cudaGetErrorString(e));
    void* base = nullptr;
    r = scratch_address(device, &base);
    if (r != RTC_OK) return r;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* d_status = (uint32_t*)base;
    rtc::WfBuffers B;
    if (NOALLOC_HEADER_BYTES + rtc_carve_wavefront((uint8_t*)base + NOALLOC_HEADER_BYTES, (uint32_t)npix, B) >
        NOALLOC_SCRATCH_BYTES)
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "path state does not fit the static scratch");
    e = cudaMemsetAsync(d_status, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, cudaGetErrorString(e));
    r = rtc_run_wavefront_sync(scene, params, B, d_status, (float4*)d_radiance_sum, st);
    if (r != RTC_OK) {
        // kernels of this call may still be queued on the stream and use the shared array: wait for
        // them, so no work of a failed call outlives it (the error recorded above is kept)
        cudaStreamSynchronize(st);
        return r;
    }
    uint32_t status = 0;
    e = cudaMemcpyAsync(&status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, cudaGetErrorString(e));
    if (status) {
        std::string m = "kernel status word " + std::to_string(status);
        return rtc_set_error((status & rtc::STATUS_TIMEOUT) ? RTC_ERR_TIMEOUT : RTC_ERR_DEVICE_CHECK, m.c_str());
    }
    return RTC_OK;
}
