// rtc_engine.h - the job-ring wavefront engine behind batched and served renders (host side).
//
// One engine owns a pool of path slots and a ring of job records on one device.  Jobs (an image of a
// scene with its own camera, resolution, spp, depth and seed) are admitted into the ring at any time;
// their pixels extend one global pixel sequence that the slots claim from, so images of different
// sizes and scenes share every extend/shade launch.  Every pixel is computed by the same per-pixel
// arithmetic as the plain render (same stream, same sample order), so a job's result does not depend
// on what else is in flight.
//
// The host drives the engine in batches of iterations on one stream and learns about progress one
// batch late (the next batch is already queued when it looks): the live slot count, the global claim
// cursor and the per-job count of finished pixels come back through pinned memory.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/rtc.h"
#include "rtc_dev.h"
#include "rtc_kernels.h"

namespace rtc {

struct EngineConfig {
    int device = 0;
    int num_sms = 148;
    uint32_t slots = 1u << 22;     // path slots (pixels in flight)
    uint32_t ring = 1024;          // job ring capacity (power of two, <= 65536)
    int mode = RTC_MODE_COMPAT;    // every job of an engine shares mode and draw order
    int draw_order = RTC_DRAW_ORDER_DEVICE;
    int batch = 12;                // iterations per batch
    uint32_t drain = 0;            // drain threshold in slots (0: 512 per SM)
    bool graphs = true;            // replay batches as a captured CUDA graph (batch a multiple of 6)
    bool wide = false;             // extend walks the 8-wide nodes (jobs asked for RTC_FLAG_WIDE_BVH)
    int block = 128;               // threads per block of the extend and shade kernels (128, 256, 512)
};

// Host view of one admitted job.
struct EngineJob {
    uint64_t seq = 0;
    uint64_t begin = 0, npix = 0;
    uint32_t nsamp = 0;
    int max_depth = 0;
    bool done = false;
    uint64_t tag = 0;              // caller's handle
    int admit_batch = 0;           // batch number at admission (older polls do not describe this job)
};

class Engine {
public:
    Engine() = default;
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;
    ~Engine();

    // Allocates the slot pool, the ring and the poll buffers on cfg.device (current device).
    rtc_status init(const EngineConfig& cfg, cudaStream_t st);
    // Starts a new run: idle slots, empty queue, empty ring.
    rtc_status reset();

    uint32_t ring_free() const { return cfg_.ring - (uint32_t)(hi_ - lo_); }
    // Stages a job for admission at the next batch (the ring must have room).  `job.begin` is set here.
    rtc_status admit(DevJob job, uint64_t tag, uint64_t* seq);
    // Enqueues one batch: the admission kernel when jobs were staged or idle slots must be refilled,
    // then `cfg.batch` (extend, shade) iterations and the poll copies.  Then waits for the poll of the
    // previous batch and updates the host view (done jobs, live slots).
    rtc_status step();
    // The drain kernel: finishes every queued slot in registers (only once all pixels are claimed).
    rtc_status finish();
    // Waits for the stream and reads the final progress (all copies complete).
    rtc_status sync_progress();

    // host view (as of the last observed poll)
    bool all_done() const { return jobs_done_ == jobs_total_; }
    bool all_claimed() const { return observed_ && next_ >= limit_; }
    uint32_t live() const { return live_; }
    uint64_t in_flight() const { return jobs_total_ - jobs_done_; }
    uint32_t observed_status() const { return status_; }   // kernel status word as of the last poll
    size_t device_bytes() const { return device_bytes_; }
    bool observed() const { return observed_; }
    uint32_t drain_threshold() const { return drain_; }
    const EngineJob& job(uint64_t seq) const { return ring_[seq & (cfg_.ring - 1)]; }
    // sequence numbers of the jobs that completed since the last call
    std::vector<uint64_t> take_completed();
    uint64_t iterations() const { return it_; }
    uint64_t launches() const { return launches_; }
    uint32_t read_status();   // kernel status word (synchronous)
    const EngineConfig& config() const { return cfg_; }
    cudaStream_t stream() const { return st_; }
    // Changes the stream of the next run (call between runs only).
    void set_stream(cudaStream_t st) { st_ = st; }
    // Instrumentation counters (8 device uint64) for the next run, or null.
    void set_counters(unsigned long long* c) { counters_ = c; }

private:
    rtc_status enqueue_admit();
    rtc_status enqueue_poll();
    rtc_status observe(int slot);
    rtc_status enqueue_iterations();
    void drop_graph();

    EngineConfig cfg_;
    cudaStream_t st_ = nullptr;
    WfTableFn fn_ = nullptr;
    WfTableFn fn_x_ = nullptr;   // the RTC_XP=1 kernels: taken once a job's scene has an xprim BVH
    void* d_wf_ = nullptr;          // slot state (carve_wavefront layout)
    WfBuffers B_{};
    DevJob* d_jobs_ = nullptr;
    uint8_t* d_prog_ = nullptr;     // WfFeed, then done[ring]
    uint32_t* d_status_ = nullptr;
    unsigned long long* counters_ = nullptr;
    DevJob* h_jobs_ = nullptr;      // pinned staging of job records
    uint8_t* h_poll_ = nullptr;     // pinned: 2 x (live count, pad, WfFeed, done[ring])
    size_t poll_bytes_ = 0;
    cudaEvent_t poll_ev_[2] = {nullptr, nullptr};
    int poll_batch_[2] = {0, 0};
    int pending_ = -1;
    int batch_no_ = 0;
    uint32_t drain_ = 0;

    std::vector<EngineJob> ring_;
    uint64_t lo_ = 0, hi_ = 0;      // jobs [lo_, hi_) are admitted and not yet observed done (lo_ oldest)
    uint64_t staged_from_ = 0;      // jobs [staged_from_, hi_) are staged, not yet published
    uint64_t limit_ = 0;            // pixels admitted (global sequence)
    uint64_t next_ = 0;             // observed claim cursor
    uint32_t live_ = 0;             // observed live slots
    uint32_t status_ = 0;           // observed kernel status word
    size_t device_bytes_ = 0;
    bool observed_ = false;
    bool refill_ = false;
    uint64_t jobs_total_ = 0, jobs_done_ = 0;
    std::vector<uint64_t> completed_;
    uint64_t it_ = 0, launches_ = 0;
    // six (extend, shade) iterations captured once: the queue rotation repeats every six iterations,
    // so the same graph serves every batch that starts at a multiple of six
    cudaGraphExec_t graph_ = nullptr;
    unsigned long long* graph_counters_ = nullptr;
};

}  // namespace rtc
