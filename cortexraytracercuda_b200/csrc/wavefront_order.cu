// wavefront_order.cu - orders the drain kernel's slots by their pixel's progress.
//
// When the wavefront hands its last slots to the drain kernel (wf_finish), each thread finishes one
// pixel's chain of bounces, and a warp runs until its longest chain ends: lanes whose pixels finish
// early sit idle (3.8 of 32 lanes active on the spheres frame).  Every slot of a single-image render
// started its pixel at iteration 0, so a slot's sample index at the drain is a measure of how long its
// samples are: few samples done means long samples and many left.  Sorting the drain queue by sample
// index puts pixels with similar remaining work in the same warps.  The order changes which thread
// finishes a pixel, never what it computes.
#include <cub/device/device_radix_sort.cuh>

#include "rtc_dev.h"
#include "rtc_internal.h"

namespace rtc {
namespace {

// keys[k] = the sample index of queue entry k (entries at or past the queue's size sort last); the
// entries are copied to `vals` for the sort to permute back into the queue
__global__ void k_order_keys(const uint32_t* __restrict__ q, const uint32_t* __restrict__ count, const uint4* meta,
                             uint32_t n_max, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t n = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_max; k += gridDim.x * blockDim.x) {
        const uint32_t slot = q[k];
        keys[k] = k < n ? meta[slot].y : 0xffffffffu;
        vals[k] = slot;
    }
}

}  // namespace
}  // namespace rtc

using namespace rtc;

size_t rtc_drain_order_temp_bytes(uint32_t max_n) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)max_n);
    return bytes;
}

cudaError_t rtc_drain_order(const WfBuffers& B, const WfIter& w, uint32_t n_max, void* temp, size_t temp_bytes,
                            cudaStream_t st) {
    if (n_max == 0 || n_max > B.slots) return cudaSuccess;
    // scratch during the drain: the hit records (two uint32 per slot) hold the keys, the long-chain
    // queue (unused once the drain starts) holds the entries being sorted
    uint32_t* keys_in = (uint32_t*)B.hit;
    uint32_t* keys_out = keys_in + B.slots;
    uint32_t* vals_in = B.queue[2];
    uint32_t* q = B.queue[w.qin];
    const int grid = (int)std::min<uint32_t>((n_max + 255) / 256, 4096u);
    k_order_keys<<<grid, 256, 0, st>>>(q, B.ctr + w.cin, B.meta, n_max, keys_in, vals_in);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t bytes = temp_bytes;
    return cub::DeviceRadixSort::SortPairs(temp, bytes, keys_in, keys_out, vals_in, q, (int)n_max, 0, 32, st);
}
