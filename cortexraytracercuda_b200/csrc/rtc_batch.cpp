// rtc_batch.cpp - rtc_render_batch: many images through one job-ring wavefront engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>

#include "rtc_engine.h"
#include "rtc_internal.h"
#include "rtc_objects.h"

using namespace rtc;

namespace {

rtc_status cuda_err(cudaError_t e, const char* what) {
    return rtc_set_error(e == cudaErrorMemoryAllocation ? RTC_ERR_OOM : RTC_ERR_CUDA,
                         (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

uint32_t next_pow2(uint32_t x) {
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

}  // namespace

// Builds the device record of one job: the scene's arrays with the job's camera and parameters.
rtc_status rtc_make_job(const rtc_scene* scene, const rtc_camera* camera, const rtc_render_params* params,
                        float* d_out, DevJob& J, void* groups) {
    J = DevJob{};
    if (groups) rtc_carve_groups(groups, params, &J.part, &J.gcnt);
    J.S = rtc_scene_view(scene, params);
    if (camera && !rtc_make_camera(*camera, J.S.cam)) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "degenerate camera");
    J.P = rtc_dev_params(params);
    J.out = (float4*)d_out;
    return RTC_OK;
}

extern "C" rtc_status rtc_render_batch(rtc_context* c, const rtc_job* jobs, uint32_t n, const rtc_batch_params* bp,
                                       void* stream) {
    if (!c || (n && !jobs)) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return RTC_OK;
    uint64_t total_pix = 0, bound = 1u << 16;
    for (uint32_t i = 0; i < n; ++i) {
        const rtc_job& j = jobs[i];
        const std::string at = "job " + std::to_string(i) + ": ";
        if (!j.scene || !j.d_radiance_sum) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, (at + "null scene or output").c_str());
        if (((uintptr_t)j.d_radiance_sum & 15u) != 0)
            return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, (at + "radiance buffer must be 16-byte aligned").c_str());
        rtc_status r = rtc_check_render_params(&j.params);
        if (r != RTC_OK) return r;
        if (j.params.mode != jobs[0].params.mode || (j.params.mode == RTC_MODE_COMPAT && j.params.draw_order != jobs[0].params.draw_order))
            return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, (at + "mode and draw order must be equal across a batch").c_str());
        if (rtc_scene_device(j.scene) != c->device)
            return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, (at + "scene lives on another device").c_str());
        const uint64_t npix = (uint64_t)j.params.width * j.params.height;
        const uint64_t sq = (uint64_t)std::max(1, (int)std::sqrt((double)j.params.spp));
        const uint64_t nsamp = j.params.mode == RTC_MODE_CLEAN ? (uint64_t)j.params.spp : sq * sq;
        total_pix += npix * (uint64_t)rtc_dev_params(&j.params).groups;
        bound += npix * nsamp * (uint64_t)(j.params.max_depth + 1);
    }
    // sample-group scratch of every image that uses it, zeroed counters (one buffer for the batch)
    std::vector<size_t> goff(n, 0);
    size_t gtotal = 0;
    for (uint32_t i = 0; i < n; ++i) {
        goff[i] = gtotal;
        gtotal += (rtc_group_bytes(&jobs[i].params) + 255) & ~(size_t)255;
    }
    EngineConfig cfg;
    cfg.device = c->device;
    cfg.num_sms = c->num_sms;
    cfg.mode = jobs[0].params.mode;
    cfg.draw_order = cfg.mode == RTC_MODE_CLEAN ? RTC_DRAW_ORDER_DEVICE : jobs[0].params.draw_order;
    // Default slots: 2^22 when a slot runs all of a pixel's samples (the batch's tail is long pixels,
    // and more slots in flight shorten it); 2^20 with sample groups, whose units are short: there the
    // path state of 2^22 slots (108 B each: the 96-byte record and the queue entries) spills out of L2,
    // and the shade kernel streams it from DRAM (64 scenes, clean mode, measured with the earlier
    // 132-byte slots: 614 Mpaths/s at 2^22, 720 at 2^20, 719 at 2^19 slots).
    const bool grouped = jobs[0].params.mode == RTC_MODE_CLEAN && (jobs[0].params.flags & RTC_FLAG_SAMPLE_GROUPS);
    cfg.slots = bp && bp->slots ? bp->slots
                                : (uint32_t)std::min<uint64_t>(total_pix, grouped ? 1u << 20 : 1u << 22);
    cfg.ring = bp && bp->ring ? bp->ring : 1024u;
    cfg.batch = bp && bp->batch > 0 ? bp->batch : 12;
    cfg.drain = bp ? bp->drain : 0u;
    cfg.wide = (jobs[0].params.flags & RTC_FLAG_WIDE_BVH) != 0;
    cfg.block = bp && bp->block ? (int)bp->block : 128;
    if (cfg.block != 128 && cfg.block != 256 && cfg.block != 512)
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "block must be 128, 256 or 512");
    if (cfg.ring != next_pow2(cfg.ring)) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "ring must be a power of two");

    std::lock_guard<std::mutex> lk(c->mu);
    RtcDeviceScope dev(c->device);
    cudaError_t e = dev.error();
    if (e != cudaSuccess) return cuda_err(e, "cudaSetDevice");
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    const EngineConfig* have = c->engine ? &c->engine->config() : nullptr;
    if (!have || have->slots != cfg.slots || have->ring != cfg.ring || have->mode != cfg.mode ||
        have->draw_order != cfg.draw_order || have->batch != cfg.batch || have->drain != cfg.drain ||
        have->wide != cfg.wide || have->block != cfg.block) {
        c->engine.reset();
        std::unique_ptr<Engine> eng(new Engine());
        rtc_status r = eng->init(cfg, st);
        if (r != RTC_OK) return r;
        c->engine = std::move(eng);
    }
    if (gtotal > c->batch_groups_cap) {
        cudaFree(c->d_batch_groups);
        c->d_batch_groups = nullptr;
        c->batch_groups_cap = 0;
        e = cudaMalloc(&c->d_batch_groups, gtotal);
        if (e != cudaSuccess) return cuda_err(e, "cudaMalloc(sample groups)");
        c->batch_groups_cap = gtotal;
    }
    if (gtotal) {
        e = cudaMemsetAsync(c->d_batch_groups, 0, gtotal, st);
        if (e != cudaSuccess) return cuda_err(e, "cudaMemsetAsync(sample groups)");
    }
    Engine& E = *c->engine;
    E.set_stream(st);
    E.set_counters(bp ? bp->d_counters : nullptr);
    rtc_status r = E.reset();
    if (r != RTC_OK) return r;

    uint32_t next_job = 0;
    bool drained = false;
    uint32_t drained_slots = 0;
    for (;;) {
        while (next_job < n && E.ring_free() > 0) {
            DevJob J;
            const rtc_job& j = jobs[next_job];
            void* g = rtc_group_bytes(&j.params) ? (uint8_t*)c->d_batch_groups + goff[next_job] : nullptr;
            r = rtc_make_job(j.scene, j.camera, &j.params, j.d_radiance_sum, J, g);
            if (r == RTC_OK) r = E.admit(J, next_job, nullptr);
            if (r != RTC_OK) return r;
            ++next_job;
        }
        r = E.step();
        if (r != RTC_OK) return r;
        if (E.observed() && next_job == n) {
            if (E.all_done()) break;
            if (E.all_claimed() && E.live() > 0 && E.live() < E.drain_threshold()) {
                drained = true;
                drained_slots = E.live();
                r = E.finish();
                if (r != RTC_OK) return r;
                break;
            }
        }
        if (E.iterations() > bound) return rtc_set_error(RTC_ERR_TIMEOUT, "batch did not complete within its iteration bound");
    }
    r = E.sync_progress();
    if (r != RTC_OK) return r;
    const uint32_t status = E.read_status();
    if (status) {
        std::string m = "kernel status word " + std::to_string(status);
        return rtc_set_error((status & STATUS_TIMEOUT) ? RTC_ERR_TIMEOUT : RTC_ERR_DEVICE_CHECK, m.c_str());
    }
    if (!E.all_done()) return rtc_set_error(RTC_ERR_DEVICE_CHECK, "batch ended with unfinished images");
    c->last = rtc_render_stats{};
    c->last.engine = RTC_ENGINE_WAVEFRONT;
    c->last.iterations = (uint32_t)E.iterations();
    c->last.launches = (uint32_t)E.launches();
    c->last.drained_slots = drained ? drained_slots : 0u;
    c->last_timed = false;
    return RTC_OK;
}
