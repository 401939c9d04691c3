// rtc_server.cpp - the render server: a request loop over the job-ring wavefront engine.
//
// Threads.  Client threads submit, poll and wait; one server thread owns the device work: it admits
// queued requests (FIFO) whenever the job ring has a free entry and the HBM budget has room for the
// request's output and, on a cache miss, its scene; it runs batches of wavefront iterations while
// anything is in flight; and when a request's last pixel is written it copies the image on a second
// stream into a reusable page-locked staging buffer (so the copy overlaps the next batches, whatever
// memory the caller's buffer is), then into the caller's buffer.
//
// Memory.  Scene slabs and request outputs come from a stream-ordered memory pool of this server
// (cudaMallocAsync / cudaFreeAsync on the server's streams), so neither admission nor eviction waits
// for the device.  A scene is evicted (least recently used first) only when no admitted request uses
// it; the kernels that used it are then already complete in stream order.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rtc_engine.h"
#include "rtc_internal.h"
#include "rtc_objects.h"

using namespace rtc;



namespace {

struct SceneEntry {
    HostScene host;
    void* d_slab = nullptr;   // resident copy, or null
    DevScene dev{};
    uint32_t refs = 0;        // admitted requests not yet complete on the device
    uint64_t last_use = 0;    // LRU clock
};

struct Request {
    uint64_t ticket = 0;
    rtc_request req{};
    float* host_out = nullptr;
    size_t out_bytes = 0;
    float4* d_out = nullptr;
    void* d_groups = nullptr;         // sample-group scratch (RTC_FLAG_SAMPLE_GROUPS)
    void* h_stage = nullptr;          // page-locked staging of the result (server-owned)
    size_t group_bytes = 0;
    cudaEvent_t copy_ev = nullptr;
    rtc_request_info info{};
    rtc_status err = RTC_OK;
    std::string err_msg;
};

}  // namespace

struct rtc_server {
    rtc_server_config cfg{};
    int num_sms = 148;
    cudaStream_t st = nullptr;        // engine stream
    cudaStream_t st_copy = nullptr;   // result copies
    cudaMemPool_t pool = nullptr;
    std::unique_ptr<Engine> eng;
    uint64_t budget = 0;
    uint64_t resident = 0;            // engine + resident scenes + outputs of admitted requests

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::vector<std::unique_ptr<SceneEntry>> scenes;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::deque<uint64_t> queue;       // tickets waiting for admission
    std::vector<uint64_t> copying;    // server thread only
    std::vector<cudaEvent_t> free_events;
    // page-locked staging buffers for result copies, reused by size: the device-to-host copy is
    // asynchronous whatever memory the caller's buffer is, and no page-locked allocation (a blocking
    // driver call) happens once the sizes in use have been seen
    std::unordered_map<size_t, std::vector<void*>> stage_free;
    std::vector<void*> stage_all;
    uint64_t next_ticket = 1;
    uint64_t lru_clock = 0;
    uint64_t in_flight = 0;           // engine jobs in flight as of the last batch (read by clients)
    bool stop = false;
    rtc_status fatal = RTC_OK;
    std::string fatal_msg;
    rtc_server_stats stats{};
    std::chrono::steady_clock::time_point t0;
    std::thread th;

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

uint64_t request_paths(const rtc_server* s, const rtc_request& r) {
    const uint64_t npix = (uint64_t)r.width * r.height;
    if (s->cfg.mode == RTC_MODE_CLEAN) return npix * (uint64_t)r.spp;
    const uint64_t sq = (uint64_t)std::sqrt((double)r.spp);
    return npix * sq * sq;
}

rtc_render_params request_params(const rtc_server* s, const rtc_request& r) {
    rtc_render_params p{};
    p.width = r.width;
    p.height = r.height;
    p.spp = r.spp;
    p.max_depth = r.max_depth;
    p.seed = r.seed;
    p.mode = s->cfg.mode;
    p.draw_order = s->cfg.draw_order;
    p.engine = RTC_ENGINE_WAVEFRONT;
    p.flags = s->cfg.flags & ~RTC_FLAG_KERNEL_TIMING;
    return p;
}

void fail_request(rtc_server* s, Request& R, rtc_status st, const std::string& msg) {
    R.err = st;
    R.err_msg = msg;
    R.info.state = RTC_REQ_FAILED;
    R.info.done_ms = s->now_ms();
    ++s->stats.failed;
}

// Marks the server broken: every queued or in-flight request fails with the message.  Caller holds mu.
void set_fatal(rtc_server* s, rtc_status st, const std::string& msg) {
    if (s->fatal == RTC_OK) {
        s->fatal = st;
        s->fatal_msg = msg;
    }
    for (auto& kv : s->reqs) {
        Request& R = *kv.second;
        if (R.info.state != RTC_REQ_DONE && R.info.state != RTC_REQ_FAILED) fail_request(s, R, st, msg);
    }
    s->queue.clear();
    s->cv_done.notify_all();
}

void note_resident(rtc_server* s) {
    s->stats.resident_bytes = s->resident;
    s->stats.peak_resident_bytes = std::max(s->stats.peak_resident_bytes, s->resident);
}

// Frees least recently used scenes that no admitted request uses, until `need` more bytes fit the
// budget (or nothing more can be evicted).  Caller holds mu.
bool make_room(rtc_server* s, uint64_t need, const SceneEntry* keep) {
    while (s->resident + need > s->budget) {
        SceneEntry* victim = nullptr;
        for (auto& e : s->scenes)
            if (e->d_slab && e->refs == 0 && e.get() != keep && (!victim || e->last_use < victim->last_use))
                victim = e.get();
        if (!victim) return false;
        cudaFreeAsync(victim->d_slab, s->st);
        victim->d_slab = nullptr;
        s->resident -= victim->host.slab.size();
        ++s->stats.scene_evictions;
    }
    return true;
}

// Admits queued requests in FIFO order while the ring and the budget allow.  Caller holds mu.
rtc_status admit_queued(rtc_server* s) {
    while (!s->queue.empty() && s->eng->ring_free() > 0) {
        Request& R = *s->reqs.at(s->queue.front());
        SceneEntry& E = *s->scenes[R.req.scene_id];
        const bool upload = E.d_slab == nullptr;
        const rtc_render_params rp = request_params(s, R.req);
        R.group_bytes = rtc_group_bytes(&rp);
        const uint64_t need = R.out_bytes + R.group_bytes + (upload ? E.host.slab.size() : 0);
        if (need + s->eng->device_bytes() > s->budget) {   // can never fit
            fail_request(s, R, RTC_ERR_OOM, "request needs more device memory than the server's HBM budget");
            s->queue.pop_front();
            s->cv_done.notify_all();
            continue;
        }
        if (!make_room(s, need, &E)) break;   // wait for requests in flight to release memory
        cudaError_t e = cudaSuccess;
        if (upload) {
            e = cudaMallocFromPoolAsync(&E.d_slab, E.host.slab.size(), s->pool, s->st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(E.d_slab, E.host.slab.data(), E.host.slab.size(), cudaMemcpyHostToDevice, s->st);
            if (e != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, (std::string("scene upload: ") + cudaGetErrorString(e)).c_str());
            E.dev = rtc_rebase_scene(E.host, (uint8_t*)E.d_slab);
            s->resident += E.host.slab.size();
            ++s->stats.scene_uploads;
        }
        void* out = nullptr;
        e = cudaMallocFromPoolAsync(&out, R.out_bytes, s->pool, s->st);
        if (e != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, (std::string("request output: ") + cudaGetErrorString(e)).c_str());
        R.d_out = (float4*)out;
        s->resident += R.out_bytes;
        DevJob J{};
        if (R.group_bytes) {
            e = cudaMallocFromPoolAsync(&R.d_groups, R.group_bytes, s->pool, s->st);
            if (e == cudaSuccess) e = cudaMemsetAsync(R.d_groups, 0, R.group_bytes, s->st);
            if (e != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, (std::string("sample groups: ") + cudaGetErrorString(e)).c_str());
            rtc_carve_groups(R.d_groups, &rp, &J.part, &J.gcnt);
            s->resident += R.group_bytes;
        }
        note_resident(s);
        J.S = E.dev;
        rtc_view_env_sampling(J.S, &rp);
        if (!R.req.use_scene_camera && !rtc_make_camera(R.req.camera, J.S.cam)) {
            cudaFreeAsync(out, s->st);
            R.d_out = nullptr;
            s->resident -= R.out_bytes;
            if (R.d_groups) {
                cudaFreeAsync(R.d_groups, s->st);
                R.d_groups = nullptr;
                s->resident -= R.group_bytes;
            }
            fail_request(s, R, RTC_ERR_INVALID_ARGUMENT, "degenerate camera");
            s->queue.pop_front();
            s->cv_done.notify_all();
            continue;
        }
        J.P = rtc_dev_params(&rp);
        J.out = R.d_out;
        rtc_status r = s->eng->admit(J, R.ticket, nullptr);
        if (r != RTC_OK) return r;
        ++E.refs;
        E.last_use = ++s->lru_clock;
        R.info.state = RTC_REQ_RUNNING;
        R.info.admit_ms = s->now_ms();
        R.info.scene_uploaded = upload ? 1 : 0;
        s->queue.pop_front();
    }
    return RTC_OK;
}

// Starts the result copy of every request whose last pixel the engine has seen written.  Caller holds mu.
rtc_status start_copies(rtc_server* s) {
    for (uint64_t seq : s->eng->take_completed()) {
        const uint64_t ticket = s->eng->job(seq).tag;
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) continue;
        Request& R = *it->second;
        SceneEntry& E = *s->scenes[R.req.scene_id];
        --E.refs;
        cudaEvent_t ev = nullptr;
        if (!s->free_events.empty()) {
            ev = s->free_events.back();
            s->free_events.pop_back();
        } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            return rtc_set_error(RTC_ERR_CUDA, "cudaEventCreate");
        }
        std::vector<void*>& fl = s->stage_free[R.out_bytes];
        if (!fl.empty()) {
            R.h_stage = fl.back();
            fl.pop_back();
        } else {
            if (cudaMallocHost(&R.h_stage, R.out_bytes) != cudaSuccess) return rtc_set_error(RTC_ERR_OOM, "cudaMallocHost(result staging)");
            s->stage_all.push_back(R.h_stage);
        }
        // the poll that reported the job complete has been waited for, so its pixels are final
        cudaError_t e = cudaMemcpyAsync(R.h_stage, R.d_out, R.out_bytes, cudaMemcpyDeviceToHost, s->st_copy);
        if (e == cudaSuccess) e = cudaEventRecord(ev, s->st_copy);
        if (e == cudaSuccess) e = cudaFreeAsync(R.d_out, s->st_copy);
        if (e == cudaSuccess && R.d_groups) {   // every pixel is final: the group scratch is free
            e = cudaFreeAsync(R.d_groups, s->st_copy);
            R.d_groups = nullptr;
            s->resident -= R.group_bytes;
        }
        if (e != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, (std::string("result copy: ") + cudaGetErrorString(e)).c_str());
        R.d_out = nullptr;
        R.copy_ev = ev;
        R.info.state = RTC_REQ_COPYING;
        s->copying.push_back(ticket);
    }
    return RTC_OK;
}

// Completes requests whose result copy has finished.  Caller holds mu.
void finish_copies(rtc_server* s) {
    size_t keep = 0;
    for (size_t i = 0; i < s->copying.size(); ++i) {
        const uint64_t t = s->copying[i];
        Request& R = *s->reqs.at(t);
        if (cudaEventQuery(R.copy_ev) != cudaSuccess) {
            s->copying[keep++] = t;
            continue;
        }
        s->free_events.push_back(R.copy_ev);
        R.copy_ev = nullptr;
        std::memcpy(R.host_out, R.h_stage, R.out_bytes);   // into the caller's buffer
        s->stage_free[R.out_bytes].push_back(R.h_stage);
        R.h_stage = nullptr;
        R.info.state = RTC_REQ_DONE;
        R.info.done_ms = s->now_ms();
        s->resident -= R.out_bytes;
        ++s->stats.completed;
        s->stats.paths += R.info.paths;
        s->cv_done.notify_all();
    }
    s->copying.resize(keep);
    note_resident(s);
}

void server_loop(rtc_server* s) {
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (s->fatal == RTC_OK) {
            rtc_status r = admit_queued(s);
            if (r != RTC_OK) set_fatal(s, r, rtc_last_error_string());
        }
        const bool busy = s->fatal == RTC_OK && s->eng->in_flight() > 0;
        if (!busy && s->copying.empty()) {
            if (s->stop) break;
            if (s->queue.empty() || s->fatal != RTC_OK) s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
            else s->cv_work.wait_for(lk, std::chrono::microseconds(200));   // waiting for memory
            continue;
        }
        if (busy) {
            lk.unlock();
            rtc_status r = s->eng->step();   // enqueues a batch, then reads the previous batch's poll
            lk.lock();
            if (r == RTC_OK && s->eng->observed_status() != 0)
                r = rtc_set_error(RTC_ERR_DEVICE_CHECK,
                                  ("kernel status word " + std::to_string(s->eng->observed_status())).c_str());
            if (r == RTC_OK) r = start_copies(s);
            if (r != RTC_OK) set_fatal(s, r, rtc_last_error_string());
            s->stats.iterations = s->eng->iterations();
            s->stats.launches = s->eng->launches();
            s->in_flight = s->eng->in_flight();
        } else if (!s->copying.empty()) {
            cudaEvent_t ev = s->reqs.at(s->copying.front())->copy_ev;
            lk.unlock();
            cudaEventSynchronize(ev);
            lk.lock();
        }
        finish_copies(s);
    }
    // stopping: nothing is in flight any more
    cudaStreamSynchronize(s->st_copy);
    cudaStreamSynchronize(s->st);
}

}  // namespace

extern "C" rtc_status rtc_server_create(const rtc_server_config* cfg, rtc_server** out) {
    if (!cfg || !out) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (cfg->mode != RTC_MODE_COMPAT && cfg->mode != RTC_MODE_CLEAN) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "unknown mode");
    if (cfg->draw_order != RTC_DRAW_ORDER_DEVICE && cfg->draw_order != RTC_DRAW_ORDER_HOST)
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "unknown draw order");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return rtc_set_error(RTC_ERR_NO_DEVICE, "no CUDA device available");
    if (cfg->device < 0 || cfg->device >= n) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "device index out of range");
    if (cfg->bvh_builder != RTC_BVH_SAH && cfg->bvh_builder != RTC_BVH_DEVICE && cfg->bvh_builder != RTC_BVH_DEVICE_LBVH)
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "unknown BVH builder");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, "cudaGetDeviceProperties");
    if (prop.major < 10) return rtc_set_error(RTC_ERR_NO_DEVICE, (std::string("device is not sm_100: ") + prop.name).c_str());
    RtcDeviceScope dev(cfg->device);
    if (dev.error() != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, "cudaSetDevice");
    std::unique_ptr<rtc_server> s(new (std::nothrow) rtc_server());
    if (!s) return rtc_set_error(RTC_ERR_OOM, "host allocation failed");
    s->cfg = *cfg;
    if (s->cfg.mode == RTC_MODE_CLEAN) s->cfg.draw_order = RTC_DRAW_ORDER_DEVICE;
    s->num_sms = prop.multiProcessorCount;
    s->budget = cfg->hbm_budget_bytes ? cfg->hbm_budget_bytes : 120ull * 1000 * 1000 * 1000;
    s->t0 = std::chrono::steady_clock::now();
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->st_copy, cudaStreamNonBlocking) != cudaSuccess)
        return rtc_set_error(RTC_ERR_CUDA, "cudaStreamCreate");
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = cfg->device;
    if (cudaMemPoolCreate(&s->pool, &pp) != cudaSuccess) return rtc_set_error(RTC_ERR_CUDA, "cudaMemPoolCreate");
    uint64_t keep = UINT64_MAX;   // keep freed blocks for reuse instead of returning them at each sync
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    EngineConfig ec;
    ec.device = cfg->device;
    ec.num_sms = s->num_sms;
    ec.slots = cfg->slots ? cfg->slots : (1u << 20);
    ec.ring = cfg->ring ? cfg->ring : 1024u;
    ec.mode = s->cfg.mode;
    ec.draw_order = s->cfg.draw_order;
    ec.batch = cfg->batch > 0 ? cfg->batch : 12;
    s->eng.reset(new (std::nothrow) Engine());
    if (!s->eng) return rtc_set_error(RTC_ERR_OOM, "host allocation failed");
    rtc_status r = s->eng->init(ec, s->st);
    if (r != RTC_OK) return r;
    s->resident = s->eng->device_bytes();
    if (s->resident > s->budget) return rtc_set_error(RTC_ERR_OOM, "path slots alone exceed the HBM budget");
    note_resident(s.get());
    rtc_server* raw = s.get();
    s->th = std::thread(server_loop, raw);
    *out = s.release();
    return RTC_OK;
}

extern "C" rtc_status rtc_server_destroy(rtc_server* s) {
    if (!s) return RTC_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (uint64_t t : s->queue) fail_request(s, *s->reqs.at(t), RTC_ERR_NOT_FOUND, "server stopped");
        s->queue.clear();
        s->cv_work.notify_all();
        s->cv_done.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    RtcDeviceScope dev(s->cfg.device);
    for (auto& e : s->scenes)
        if (e->d_slab) cudaFreeAsync(e->d_slab, s->st);
    for (auto& kv : s->reqs) {
        if (kv.second->d_out) cudaFreeAsync(kv.second->d_out, s->st);
        if (kv.second->d_groups) cudaFreeAsync(kv.second->d_groups, s->st);
        if (kv.second->copy_ev) cudaEventDestroy(kv.second->copy_ev);
    }
    cudaStreamSynchronize(s->st);
    for (cudaEvent_t e : s->free_events) cudaEventDestroy(e);
    for (void* h : s->stage_all) cudaFreeHost(h);
    s->eng.reset();   // the engine's buffers are released before the streams go
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->st_copy) cudaStreamDestroy(s->st_copy);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
    return RTC_OK;
}

extern "C" rtc_status rtc_server_add_scene(rtc_server* s, const rtc_scene_desc* desc, uint32_t* scene_id) {
    if (!s || !desc || !scene_id) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_ptr<SceneEntry> e(new (std::nothrow) SceneEntry());
    if (!e) return rtc_set_error(RTC_ERR_OOM, "host allocation failed");
    rtc_status r = rtc_build_host_scene(desc, e->host, s->cfg.bvh_builder, s->cfg.device);   // outside the lock
    if (r != RTC_OK) return r;
    std::lock_guard<std::mutex> lk(s->mu);
    *scene_id = (uint32_t)s->scenes.size();
    s->scenes.push_back(std::move(e));
    return RTC_OK;
}

extern "C" rtc_status rtc_server_submit(rtc_server* s, const rtc_request* req, float* radiance_sum, uint64_t* ticket) {
    if (!s || !req || !radiance_sum || !ticket) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_ptr<Request> R(new (std::nothrow) Request());
    if (!R) return rtc_set_error(RTC_ERR_OOM, "host allocation failed");
    R->req = *req;
    const rtc_render_params p = request_params(s, *req);
    rtc_status r = rtc_check_render_params(&p);
    if (r != RTC_OK) return r;
    R->host_out = radiance_sum;
    R->out_bytes = (size_t)req->width * req->height * sizeof(float4);
    R->info.paths = request_paths(s, *req);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "server is stopping");
    if (s->fatal != RTC_OK) return rtc_set_error(s->fatal, s->fatal_msg.c_str());
    if (req->scene_id >= s->scenes.size()) return rtc_set_error(RTC_ERR_NOT_FOUND, "unknown scene id");
    R->ticket = s->next_ticket++;
    R->info.state = RTC_REQ_QUEUED;
    R->info.submit_ms = s->now_ms();
    *ticket = R->ticket;
    s->queue.push_back(R->ticket);
    s->reqs.emplace(R->ticket, std::move(R));
    ++s->stats.submitted;
    s->cv_work.notify_one();
    return RTC_OK;
}

namespace {
// Reports a request's state; releases it when it is finished.  Caller holds mu.
rtc_status report(rtc_server* s, uint64_t ticket, rtc_request_info* info) {
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return rtc_set_error(RTC_ERR_NOT_FOUND, "unknown ticket");
    Request& R = *it->second;
    if (info) *info = R.info;
    if (R.info.state == RTC_REQ_DONE) {
        s->reqs.erase(it);
        return RTC_OK;
    }
    if (R.info.state == RTC_REQ_FAILED) {
        rtc_status e = R.err;
        std::string m = R.err_msg;
        s->reqs.erase(it);
        return rtc_set_error(e, m.c_str());
    }
    return RTC_ERR_BUSY;
}
}  // namespace

extern "C" rtc_status rtc_server_poll(rtc_server* s, uint64_t ticket, rtc_request_info* info) {
    if (!s) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    rtc_status r = report(s, ticket, info);
    if (r == RTC_ERR_BUSY) rtc_set_error(RTC_ERR_BUSY, "request in flight");
    return r;
}

extern "C" rtc_status rtc_server_wait(rtc_server* s, uint64_t ticket, int32_t timeout_ms, rtc_request_info* info) {
    if (!s) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
    for (;;) {
        rtc_status r = report(s, ticket, info);
        if (r != RTC_ERR_BUSY) return r;
        if (timeout_ms < 0) {
            s->cv_done.wait(lk);
        } else if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout) {
            r = report(s, ticket, info);
            if (r != RTC_ERR_BUSY) return r;
            return rtc_set_error(RTC_ERR_TIMEOUT, "request not done within the timeout");
        }
    }
}

extern "C" rtc_status rtc_server_get_stats(rtc_server* s, rtc_server_stats* st) {
    if (!s || !st) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->stats;
    st->queued = (uint32_t)s->queue.size();
    st->in_flight = (uint32_t)(s->in_flight + s->copying.size());
    return RTC_OK;
}
