// rtc_engine.cpp - the job-ring wavefront engine (host driver).
#include "rtc_engine.h"

#include <algorithm>
#include <cstring>
#include <string>

#include "rtc_internal.h"

namespace rtc {

namespace {

constexpr size_t POLL_LIVE = 0;                 // uint32 live slots
constexpr size_t POLL_STATUS = 4;               // uint32 kernel status word
constexpr size_t POLL_FEED = 8;                 // WfFeed
constexpr size_t POLL_DONE = 8 + sizeof(WfFeed);   // uint32 done[ring]

rtc_status cuda_err(cudaError_t e, const char* what) {
    return rtc_set_error(e == cudaErrorMemoryAllocation ? RTC_ERR_OOM : RTC_ERR_CUDA,
                         (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

#define ENG_CUDA(call)                                      \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_err(_e, #call);  \
    } while (0)

}  // namespace

Engine::~Engine() {
    if (st_) cudaStreamSynchronize(st_);
    drop_graph();
    cudaFree(d_wf_);
    cudaFree(d_jobs_);
    cudaFree(d_prog_);
    cudaFree(d_status_);
    if (h_jobs_) cudaFreeHost(h_jobs_);
    if (h_poll_) cudaFreeHost(h_poll_);
    for (cudaEvent_t e : poll_ev_)
        if (e) cudaEventDestroy(e);
}

rtc_status Engine::init(const EngineConfig& cfg, cudaStream_t st) {
    if (cfg.ring == 0 || (cfg.ring & (cfg.ring - 1)) != 0 || cfg.ring > WF_MAX_JOBS)
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "job ring size must be a power of two <= 65536");
    if (cfg.slots == 0 || cfg.slots > (1u << 24))
        return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "slot count must be in 1..2^24");
    cfg_ = cfg;
    st_ = st;
    if (cfg.mode == RTC_MODE_CLEAN) { fn_ = rtc_wf_table_clean; fn_x_ = rtc_wf_table_clean_x; }
    else if (cfg.draw_order == RTC_DRAW_ORDER_HOST) { fn_ = rtc_wf_table_compat_host; fn_x_ = rtc_wf_table_compat_host_x; }
    else { fn_ = rtc_wf_table_compat_dev; fn_x_ = rtc_wf_table_compat_dev_x; }
    drain_ = cfg.drain ? cfg.drain : (uint32_t)cfg.num_sms * 512u;
    device_bytes_ = (size_t)cfg.slots * rtc_wf_slot_bytes() + 16 * 256 + (size_t)cfg.ring * sizeof(DevJob) +
                    sizeof(WfFeed) + (size_t)cfg.ring * sizeof(uint32_t) + 256;
    ENG_CUDA(cudaMalloc(&d_wf_, (size_t)cfg.slots * rtc_wf_slot_bytes() + 16 * 256));
    rtc_carve_wavefront(d_wf_, cfg.slots, B_);
    ENG_CUDA(cudaMalloc(&d_jobs_, (size_t)cfg.ring * sizeof(DevJob)));
    ENG_CUDA(cudaMalloc(&d_prog_, sizeof(WfFeed) + (size_t)cfg.ring * sizeof(uint32_t)));
    ENG_CUDA(cudaMalloc(&d_status_, sizeof(uint32_t)));
    ENG_CUDA(cudaMallocHost(&h_jobs_, (size_t)cfg.ring * sizeof(DevJob)));
    poll_bytes_ = (POLL_DONE + (size_t)cfg.ring * sizeof(uint32_t) + 255) & ~(size_t)255;
    ENG_CUDA(cudaMallocHost(&h_poll_, 2 * poll_bytes_));
    for (cudaEvent_t& e : poll_ev_) ENG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ring_.assign(cfg.ring, EngineJob{});
    return reset();
}

rtc_status Engine::reset() {
    ENG_CUDA(cudaMemsetAsync(B_.ctr, 0, WF_CTR_N * sizeof(uint32_t), st_));
    // every slot idle (pixel word 0xffffffff); the other words are written before they are read
    ENG_CUDA(cudaMemsetAsync(B_.rec, 0xff, (size_t)cfg_.slots * WF_REC_BYTES, st_));
    ENG_CUDA(cudaMemsetAsync(d_prog_, 0, sizeof(WfFeed) + (size_t)cfg_.ring * sizeof(uint32_t), st_));
    ENG_CUDA(cudaMemsetAsync(d_status_, 0, sizeof(uint32_t), st_));
    ENG_CUDA(cudaStreamSynchronize(st_));
    std::fill(ring_.begin(), ring_.end(), EngineJob{});
    lo_ = hi_ = staged_from_ = 0;
    limit_ = next_ = 0;
    live_ = 0;
    status_ = 0;
    observed_ = false;
    refill_ = false;
    jobs_total_ = jobs_done_ = 0;
    completed_.clear();
    it_ = launches_ = 0;
    pending_ = -1;
    batch_no_ = 0;
    return RTC_OK;
}

rtc_status Engine::admit(DevJob job, uint64_t tag, uint64_t* seq) {
    if (ring_free() == 0) return rtc_set_error(RTC_ERR_BUSY, "job ring is full");
    if (job.S.num_xnodes && fn_ != fn_x_) {   // from now on the kernels that also walk xprim BVHs
        fn_ = fn_x_;
        drop_graph();
    }
    const uint64_t s = hi_++;
    const uint32_t slot = (uint32_t)(s & (cfg_.ring - 1));
    const uint64_t npix = (uint64_t)job.P.num_pixels;
    job.begin = limit_;
    limit_ += npix * (uint64_t)std::max(1, job.P.groups);   // work units: pixel x sample group
    h_jobs_[slot] = job;
    ENG_CUDA(cudaMemcpyAsync(d_jobs_ + slot, h_jobs_ + slot, sizeof(DevJob), cudaMemcpyHostToDevice, st_));
    uint32_t* d_done = (uint32_t*)(d_prog_ + sizeof(WfFeed));
    ENG_CUDA(cudaMemsetAsync(d_done + slot, 0, sizeof(uint32_t), st_));
    EngineJob& J = ring_[slot];
    J = EngineJob{};
    J.seq = s;
    J.begin = job.begin;
    J.npix = npix;
    J.nsamp = cfg_.mode == RTC_MODE_CLEAN ? (uint32_t)job.P.spp : (uint32_t)(job.P.sqrt_spp * job.P.sqrt_spp);
    J.max_depth = job.P.max_depth;
    J.tag = tag;
    J.admit_batch = batch_no_;
    ++jobs_total_;
    if (seq) *seq = s;
    return RTC_OK;
}

rtc_status Engine::enqueue_admit() {
    WfTableArgs A{d_jobs_, (WfFeed*)d_prog_, (uint32_t*)(d_prog_ + sizeof(WfFeed)), cfg_.ring - 1};
    WfLaunch L{};
    L.w = wf_iter(it_);
    L.win.limit = limit_;
    L.win.lo = (uint32_t)lo_;
    L.win.hi = (uint32_t)hi_;
    L.status = d_status_;
    L.st = st_;
    L.grid = (int)std::min<uint64_t>((cfg_.slots + 127) / 128, (uint64_t)cfg_.num_sms * 16);
    cudaError_t e = fn_(WF_OP_ADMIT, A, B_, L);
    if (e != cudaSuccess) return cuda_err(e, "job admission");
    launches_ += 2;   // window update + admission
    staged_from_ = hi_;
    refill_ = false;
    return RTC_OK;
}

rtc_status Engine::enqueue_poll() {
    const int slot = batch_no_ & 1;
    uint8_t* h = h_poll_ + (size_t)slot * poll_bytes_;
    ENG_CUDA(cudaMemcpyAsync(h + POLL_LIVE, B_.ctr + wf_iter(it_).cin, sizeof(uint32_t), cudaMemcpyDeviceToHost, st_));
    ENG_CUDA(cudaMemcpyAsync(h + POLL_STATUS, d_status_, sizeof(uint32_t), cudaMemcpyDeviceToHost, st_));
    ENG_CUDA(cudaMemcpyAsync(h + POLL_FEED, d_prog_, sizeof(WfFeed) + (size_t)cfg_.ring * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, st_));
    ENG_CUDA(cudaEventRecord(poll_ev_[slot], st_));
    poll_batch_[slot] = batch_no_;
    return RTC_OK;
}

rtc_status Engine::observe(int slot) {
    const uint8_t* h = h_poll_ + (size_t)slot * poll_bytes_;
    const int pb = poll_batch_[slot];
    uint32_t live = 0;
    WfFeed feed;
    std::memcpy(&live, h + POLL_LIVE, sizeof live);
    std::memcpy(&status_, h + POLL_STATUS, sizeof status_);
    std::memcpy(&feed, h + POLL_FEED, sizeof feed);
    const uint32_t* done = (const uint32_t*)(h + POLL_DONE);
    live_ = live;
    next_ = feed.next;
    for (uint64_t s = lo_; s < hi_; ++s) {
        EngineJob& J = ring_[s & (cfg_.ring - 1)];
        // a counter copied before the job's admission may still hold the previous occupant's count
        if (J.done || J.admit_batch > pb) continue;
        if (done[s & (cfg_.ring - 1)] >= J.npix) {
            J.done = true;
            ++jobs_done_;
            completed_.push_back(s);
        }
    }
    while (lo_ < hi_ && ring_[lo_ & (cfg_.ring - 1)].done) ++lo_;
    observed_ = true;
    // no live slot while work is unfinished: idle slots must claim the remaining pixels
    if (live_ == 0 && jobs_done_ < jobs_total_) refill_ = true;
    return RTC_OK;
}

void Engine::drop_graph() {
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
}

rtc_status Engine::enqueue_iterations() {
    WfTableArgs A{d_jobs_, (WfFeed*)d_prog_, (uint32_t*)(d_prog_ + sizeof(WfFeed)), cfg_.ring - 1};
    WfLaunch L{};
    L.status = d_status_;
    L.counters = counters_;
    L.wide = cfg_.wide;
    // a batch mixes scenes of every size: its walks are uneven, and warps take queue chunks from a
    // counter (64 scenes: compat 873 -> 997 Mpaths/s, clean with sample groups 834 -> 985, against
    // the fixed grid stride)
    L.dynamic = rtc_dynamic_chunks(true);
    L.block = cfg_.block;
    L.grid = cfg_.num_sms * 8 * 128 / cfg_.block;   // 1,024 threads per SM
    const bool use_graph = cfg_.graphs && st_ != nullptr && cfg_.batch % 6 == 0 && it_ % 6 == 0;
    if (use_graph && (!graph_ || graph_counters_ != counters_)) {
        drop_graph();
        cudaGraph_t g = nullptr;
        ENG_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        L.st = st_;
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < 6 && e == cudaSuccess; ++k) {
            L.w = wf_iter((uint64_t)k);
            e = fn_(WF_OP_EXTEND, A, B_, L);
            if (e == cudaSuccess) e = fn_(WF_OP_SHADE, A, B_, L);
        }
        cudaError_t e2 = cudaStreamEndCapture(st_, &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&graph_, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {   // capture unavailable here: launch directly from now on
            graph_ = nullptr;
            cfg_.graphs = false;
            cudaGetLastError();
        } else {
            graph_counters_ = counters_;
        }
    }
    if (use_graph && graph_) {
        for (int k = 0; k < cfg_.batch; k += 6) ENG_CUDA(cudaGraphLaunch(graph_, st_));
        it_ += (uint64_t)cfg_.batch;
        launches_ += 2u * (uint64_t)cfg_.batch;
        return RTC_OK;
    }
    L.st = st_;
    for (int k = 0; k < cfg_.batch; ++k, ++it_) {
        L.w = wf_iter(it_);
        cudaError_t e = fn_(WF_OP_EXTEND, A, B_, L);
        if (e == cudaSuccess) e = fn_(WF_OP_SHADE, A, B_, L);
        if (e != cudaSuccess) return cuda_err(e, "wavefront iteration");
        launches_ += 2;
    }
    return RTC_OK;
}

rtc_status Engine::step() {
    if (staged_from_ < hi_ || refill_) {
        rtc_status r = enqueue_admit();
        if (r != RTC_OK) return r;
    }
    rtc_status r = enqueue_iterations();
    if (r != RTC_OK) return r;
    r = enqueue_poll();
    if (r != RTC_OK) return r;
    const int slot = batch_no_ & 1;
    ++batch_no_;
    if (pending_ >= 0) {
        ENG_CUDA(cudaEventSynchronize(poll_ev_[pending_]));
        r = observe(pending_);
        if (r != RTC_OK) return r;
    }
    pending_ = slot;
    return RTC_OK;
}

rtc_status Engine::finish() {
    WfTableArgs A{d_jobs_, (WfFeed*)d_prog_, (uint32_t*)(d_prog_ + sizeof(WfFeed)), cfg_.ring - 1};
    WfLaunch L{};
    L.w = wf_iter(it_);
    L.status = d_status_;
    L.counters = counters_;
    L.wide = cfg_.wide;
    L.st = st_;
    L.drain_every = rtc_drain_every(0);   // the batch's drain is its tail of long chains: the plain drain
    const uint32_t per_block = L.drain_every > 0 ? (uint32_t)WF_DRAIN_BLOCK : 128u;
    L.grid = (int)std::max<uint32_t>(1u, (drain_ + per_block - 1u) / per_block);
    cudaError_t e = fn_(WF_OP_FINISH, A, B_, L);
    if (e != cudaSuccess) return cuda_err(e, "wavefront finish");
    ++launches_;
    return RTC_OK;
}

rtc_status Engine::sync_progress() {
    if (staged_from_ < hi_) {   // publish staged jobs first so the final view covers them
        rtc_status r = enqueue_admit();
        if (r != RTC_OK) return r;
    }
    rtc_status r = enqueue_poll();
    if (r != RTC_OK) return r;
    const int slot = batch_no_ & 1;
    ++batch_no_;
    ENG_CUDA(cudaStreamSynchronize(st_));
    pending_ = -1;
    return observe(slot);
}

std::vector<uint64_t> Engine::take_completed() {
    std::vector<uint64_t> out;
    out.swap(completed_);
    return out;
}

uint32_t Engine::read_status() {
    uint32_t s = 0;
    if (cudaMemcpyAsync(&s, d_status_, sizeof s, cudaMemcpyDeviceToHost, st_) != cudaSuccess) return 0xffffffffu;
    if (cudaStreamSynchronize(st_) != cudaSuccess) return 0xffffffffu;
    return s;
}

}  // namespace rtc
