// bvh_build.h - host SAH BVH2 builder producing the flattened 64-byte node layout of rtc_dev.h.
//
// Replaces the reference's bvh_node constructor (core/src/misc/bvh_node.cuh:63-108), which picks a
// random axis with one RNG draw, exchange-sorts the span (O(n^2)) and splits at the median on a single
// device thread.  Here: binned SAH (32 bins over the centroid bounds) on the host, leaves of at most
// `max_leaf` items, subtrees built in parallel with std::thread.  Closest-hit results do not depend
// on the tree, only the order in which exactly-equal-t candidates are met does.
#pragma once

#include <stdint.h>

#include <vector>

namespace rtc {

struct Aabb {
    float lo[3], hi[3];
};

struct BvhInput {
    std::vector<Aabb> boxes;       // one per primitive (already padded)
};

struct BvhOutput {
    std::vector<float> nodes;      // 16 floats per node (4 x float4), see rtc_dev.h
    std::vector<float> nodes8;     // the same tree collapsed to 8-wide nodes with quantised child boxes:
                                   // NODE8_FLOATS (5 x float4) per node, see rtc_dev.h; same leaves
    std::vector<uint32_t> items8;  // the 8-wide nodes' leaf ranges: per entry, a position in `order`
    std::vector<uint32_t> order;   // primitive index per leaf slot, leaf order
    uint32_t num_nodes = 0;
    uint32_t num_nodes8 = 0;
    uint32_t max_depth = 0;
    uint32_t max_leaf_seen = 0;
};

// Returns false (with a message) if the tree would not fit the traversal stack or the item encoding.
bool build_bvh(const BvhInput& in, int max_leaf, int threads, BvhOutput& out, const char** err);

// Merges subtrees of at most `max_leaf` primitives into single leaves where the SAH cost favours it
// (bvh_build.cpp): renumbers the nodes depth-first and reorders `order` so each leaf is contiguous;
// updates num_nodes, max_depth and max_leaf_seen.  For one-primitive-per-leaf trees.
void collapse_leaves(BvhOutput& tree, int max_leaf);

// BVH built on CUDA device `device` (bvh_device.cu) over Morton-sorted primitives, one primitive per
// leaf, no 8-wide nodes: PLOC clustering (BVH_DEVICE_PLOC) or the linear BVH (BVH_DEVICE_LBVH).
// BVH_DEVICE_TOO_DEEP and BVH_DEVICE_UNSUPPORTED leave the SAH build as the way out.
enum BvhDeviceStatus { BVH_DEVICE_OK = 0, BVH_DEVICE_TOO_DEEP = 1, BVH_DEVICE_UNSUPPORTED = 2, BVH_DEVICE_ERROR = 3 };
enum BvhDeviceMethod { BVH_DEVICE_PLOC = 0, BVH_DEVICE_LBVH = 1 };
int build_bvh_device(const BvhInput& in, int device, BvhDeviceMethod method, BvhOutput& out, const char** err);

}  // namespace rtc
