// rtc_objects.h - the opaque handles of the C ABI (host side, shared by the ABI translation units).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/rtc.h"
#include "rtc_dev.h"
#include "rtc_engine.h"

struct rtc_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t* d_status = nullptr;
    unsigned long long* d_counters = nullptr;
    float4* d_out = nullptr;
    size_t out_cap = 0;         // float4 elements
    uint8_t* d_rgb8 = nullptr;
    size_t rgb8_cap = 0;
    int num_sms = 148;
    // wavefront scratch: path slot records and the slot queues (carve_wavefront)
    void* d_wf = nullptr;
    uint32_t wf_cap = 0;
    void* d_groups = nullptr;          // sample-group partial sums and counters (RTC_FLAG_SAMPLE_GROUPS)
    size_t groups_cap = 0;
    void* d_batch_groups = nullptr;    // the same for the images of a batch
    size_t batch_groups_cap = 0;
    uint32_t* h_poll = nullptr;       // pinned: queue sizes read back between batches
    cudaEvent_t poll_ev[2] = {nullptr, nullptr};
    cudaEvent_t phase_ev[3] = {nullptr, nullptr, nullptr};   // render start, drain start, render end
    cudaStream_t stream_long = nullptr;    // the long-chain drain kernel, beside the bulk iterations
    cudaEvent_t split_ev[2] = {nullptr, nullptr};
    rtc_render_stats last{};
    bool last_timed = false;
    std::vector<cudaEvent_t> kev;      // per-launch timing events (RTC_FLAG_KERNEL_TIMING)
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> kev_pairs;   // extend pairs, then shade pairs
    uint32_t kev_ext = 0, kev_shade = 0;   // pairs used by the last render
    std::unique_ptr<rtc::Engine> engine;   // job-ring engine of rtc_render_batch (created on first use)
    std::mutex mu;
};

struct rtc_scene {
    rtc_context* ctx = nullptr;   // creating context; not dereferenced after creation
    int device = 0;
    void* d_slab = nullptr;
    size_t slab_bytes = 0;
    rtc::DevScene dev{};
    rtc_camera cam{};
    rtc_scene_info info{};
};


// Host image of a scene: the flattened device slab (BVH, primitives, materials, textures, images,
// environment map) built once on the host, uploadable to any device address.  Pointer fields of `dev`
// hold byte offsets into `slab`.
struct HostScene {
    std::vector<uint8_t> slab;
    rtc::DevScene dev{};
    rtc_camera cam{};
    rtc_scene_info info{};
};
// Validates and flattens a scene description, building its BVH (the work of rtc_scene_create before
// the upload).
// `bvh_builder` is an RTC_BVH_* value; RTC_BVH_DEVICE builds on CUDA device `device`.
rtc_status rtc_build_host_scene(const rtc_scene_desc* d, HostScene& out, uint32_t bvh_builder = 0, int device = 0);
// The DevScene of a host scene whose slab was copied to `base`.
rtc::DevScene rtc_rebase_scene(const HostScene& h, uint8_t* base);
