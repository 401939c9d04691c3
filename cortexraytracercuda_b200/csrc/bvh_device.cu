// bvh_device.cu - device BVH build (linear BVH over Morton codes) for rtc_scene_create_ex.
//
// The reference builds its BVH on one device thread, choosing a random axis per node and
// exchange-sorting the span (O(n^2), core/src/misc/bvh_node.cuh:63-108, called from gpu.cu:749).  The
// library's default is a binned SAH build on host threads (bvh_build.cpp); this is the fast
// alternative for large meshes and cache misses, in the layout the traversal already reads:
//   1. 30-bit Morton code of each primitive's box centroid (10 bits per axis over the centroid bounds);
//   2. radix sort of (code, primitive) pairs (CUB);
//   3. one thread per internal node finds the node's key range and split from the longest common
//      prefixes of neighbouring codes (Karras, "Maximizing Parallelism in the Construction of BVHs,
//      Octrees, and k-d Trees", HPG 2012), ties between equal codes broken by sorted position;
//   4. bottom-up boxes: every leaf walks towards the root; the first thread to reach a node stops, the
//      second (both children now known) writes the node's 64-byte record and goes on - no thread ever
//      waits for another.
// The tree comes out with one primitive per leaf in sorted order (a host pass, collapse_leaves, can
// merge small subtrees into leaves by SAH cost; see RTC_DEVICE_LEAF_MAX).  Quality is below the SAH
// build's (more node visits per ray); the build is a few milliseconds where the host build of a million
// triangles takes a second.
//
// The default device method replaces steps 3-4 with PLOC (Meister and Bittner, "Parallel Locally-Ordered
// Clustering for Bounding Volume Hierarchy Construction", IEEE TVCG 2018): starting from the sorted
// primitives as clusters, each round finds every cluster's nearest neighbour among the PLOC_RADIUS
// clusters on either side (the one whose union box has the smallest surface area, the smaller position
// on a tie), merges mutual nearest neighbours into a new node, and compacts the survivors in order.
// Merging by the surface-area distance gives trees close to a SAH build's.  Node indices count down from
// the round's cluster count, so the last merge - the root - is node 0, and the numbering is
// deterministic (a prefix sum orders each round's merges).  PLOC stops at RTC_PLOC_TOP clusters; the
// host's binned SAH build joins those into the top of the tree (join_top).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <vector>

#include "bvh_build.h"
#include "rtc_dev.h"
#include "rtc_internal.h"

// Largest leaf of the device-built trees after the SAH collapse (a build-time knob).  The default, 1,
// keeps one primitive per leaf as the builders make them: on the meshes frame (1.31 M triangles, PLOC)
// leaves of up to 4 cut node visits by 5% (15.04 -> 14.26 G) but the frame measured 1% slower (361 against
// 366 Mpaths/s); the gap to the SAH tree (395 Mpaths/s, 12.61 G visits) is in its upper levels.
#ifndef RTC_DEVICE_LEAF_MAX
#define RTC_DEVICE_LEAF_MAX 1
#endif
// PLOC stops at this many clusters, and the host's binned SAH build joins them (a build-time knob; 1:
// PLOC all the way to the root).  Meshes frame (1.31 M triangles), against 392.7-394.4 Mpaths/s with the
// host SAH tree: PLOC to the root 367.8, joined at 4,096 clusters 381.1, at 32,768 380.6-383.4, at
// 131,072 385.7; the join adds about 50 ms (32,768) to 140 ms (131,072) to a 200 ms scene create.
#ifndef RTC_PLOC_TOP
#define RTC_PLOC_TOP 131072
#endif

namespace rtc {
namespace {

__device__ __forceinline__ uint32_t spread10(uint32_t v) {   // bit k of v -> bit 3k
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_morton(const Aabb* __restrict__ boxes, uint32_t n, float3 lo, float3 scale, uint32_t* keys,
                         uint32_t* vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Aabb b = boxes[i];
    uint32_t q[3];
    const float c[3] = {0.5f * (b.lo[0] + b.hi[0]), 0.5f * (b.lo[1] + b.hi[1]), 0.5f * (b.lo[2] + b.hi[2])};
    const float l[3] = {lo.x, lo.y, lo.z}, s[3] = {scale.x, scale.y, scale.z};
    for (int k = 0; k < 3; ++k) {
        float x = (c[k] - l[k]) * s[k];
        x = x < 0.0f ? 0.0f : (x > 1023.0f ? 1023.0f : x);
        q[k] = (uint32_t)x;
    }
    keys[i] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    vals[i] = i;
}

// Length of the common prefix of sorted keys a and b (-1 outside [0, n)); equal keys compare their
// positions, so every prefix is distinct.
__device__ __forceinline__ int delta(const uint32_t* __restrict__ k, int64_t n, int64_t a, int64_t b) {
    if (b < 0 || b >= n) return -1;
    const uint32_t ka = k[a], kb = k[b];
    if (ka == kb) return 32 + __clz((uint32_t)a ^ (uint32_t)b);
    return __clz(ka ^ kb);
}

// Children of internal node i: >= 0 an internal node, < 0 a leaf in the node layout's encoding.
__global__ void k_internal(const uint32_t* __restrict__ keys, uint32_t n, int32_t* __restrict__ child,
                           int32_t* __restrict__ parent_int, int32_t* __restrict__ parent_leaf, uint32_t* error) {
    const int64_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t N = n;
    if (i >= N - 1) return;
    const int d = delta(keys, N, i, i + 1) - delta(keys, N, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = delta(keys, N, i, i - d);
    int64_t lmax = 2;
    int guard = 0;
    while (delta(keys, N, i, i + lmax * d) > dmin) {
        lmax *= 2;
        if (++guard > 40) { atomicOr(error, 1u); return; }
    }
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2)
        if (delta(keys, N, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(keys, N, i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) / 2;
        if (delta(keys, N, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int64_t g = i + s * d + (d < 0 ? -1 : 0);
    const int64_t lo = i < j ? i : j, hi = i < j ? j : i;
    int32_t cl, cr;
    if (lo == g) {
        cl = (int32_t)~(((uint32_t)g << LEAF_COUNT_BITS) | 1u);
        parent_leaf[g] = (int32_t)i;
    } else {
        cl = (int32_t)g;
        parent_int[g] = (int32_t)i;
    }
    if (hi == g + 1) {
        cr = (int32_t)~(((uint32_t)(g + 1) << LEAF_COUNT_BITS) | 1u);
        parent_leaf[g + 1] = (int32_t)i;
    } else {
        cr = (int32_t)(g + 1);
        parent_int[g + 1] = (int32_t)i;
    }
    child[2 * i] = cl;
    child[2 * i + 1] = cr;
}

// A child's box: an inner node's box was written by another thread (possibly on another SM), so it is
// read from L2 (ld.global.cg), never from a possibly stale L1 line.
__device__ __forceinline__ Aabb box_of(int32_t c, const Aabb* __restrict__ boxes, const uint32_t* __restrict__ vals,
                                       const Aabb* node_box) {
    Aabb b;
    if (c >= 0) {
        const float* f = node_box[c].lo;
        for (int k = 0; k < 3; ++k) {
            b.lo[k] = __ldcg(f + k);
            b.hi[k] = __ldcg(f + 3 + k);
        }
        return b;
    }
    const uint32_t pos = ((uint32_t)~c) >> LEAF_COUNT_BITS;
    return boxes[vals[pos]];
}

// Bottom-up pass: writes every internal node's record (both child boxes and child links) and box, and
// the depth of the deepest leaf.
__global__ void k_bottom_up(const Aabb* __restrict__ boxes, const uint32_t* __restrict__ vals, uint32_t n,
                            const int32_t* __restrict__ child, const int32_t* __restrict__ parent_int,
                            const int32_t* __restrict__ parent_leaf, uint32_t* flags, Aabb* node_box,
                            float4* nodes, uint32_t* max_depth, uint32_t* error) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    // Every index read from the link arrays is range-checked (they start as -1): a malformed tree sets
    // an error bit instead of reading out of bounds.
    const int32_t inner = (int32_t)n - 1;
    auto inner_ok = [inner](int32_t p) { return p >= 0 && p < inner; };
    // depth of this leaf
    uint32_t depth = 1;
    int32_t p = parent_leaf[k];
    if (!inner_ok(p)) { atomicOr(error, 2u); return; }
    while (p != 0) {
        p = parent_int[p];
        if (++depth > 4096u || !inner_ok(p)) { atomicOr(error, 2u); return; }
    }
    atomicMax(max_depth, depth + 1u);
    int32_t node = parent_leaf[k];
    for (uint32_t steps = 0; steps < 4096u; ++steps) {
        __threadfence();
        if (atomicAdd(flags + node, 1u) == 0u) return;   // the other child is not done yet: it goes on
        __threadfence();
        const int32_t cl = child[2 * node], cr = child[2 * node + 1];
        const bool okl = cl >= 0 ? cl < inner : (((uint32_t)~cl) >> LEAF_COUNT_BITS) < n;
        const bool okr = cr >= 0 ? cr < inner : (((uint32_t)~cr) >> LEAF_COUNT_BITS) < n;
        if (!okl || !okr) { atomicOr(error, 8u); return; }
        const Aabb L = box_of(cl, boxes, vals, node_box), R = box_of(cr, boxes, vals, node_box);
        Aabb U;
        for (int a = 0; a < 3; ++a) {
            U.lo[a] = fminf(L.lo[a], R.lo[a]);
            U.hi[a] = fmaxf(L.hi[a], R.hi[a]);
        }
        node_box[node] = U;
        float4* np = nodes + 4 * (size_t)node;
        np[0] = make_float4(L.lo[0], L.hi[0], L.lo[1], L.hi[1]);
        np[1] = make_float4(R.lo[0], R.hi[0], R.lo[1], R.hi[1]);
        np[2] = make_float4(L.lo[2], L.hi[2], R.lo[2], R.hi[2]);
        np[3] = make_float4(__int_as_float(cl), __int_as_float(cr), 0.0f, 0.0f);
        if (node == 0) return;
        node = parent_int[node];
        if (!inner_ok(node)) { atomicOr(error, 8u); return; }
    }
    atomicOr(error, 4u);
}

// ---- PLOC ---------------------------------------------------------------------------------------
constexpr int PLOC_RADIUS = 16;
constexpr int PLOC_BLOCK = 256;
constexpr int PLOC_MAX_ROUNDS = 512;

struct Cluster {
    Aabb box;
    int32_t id;   // >= 0 inner node, < 0 leaf in the node layout's encoding
};

__device__ __forceinline__ Aabb unite(const Aabb& a, const Aabb& b) {
    Aabb u;
    for (int k = 0; k < 3; ++k) {
        u.lo[k] = fminf(a.lo[k], b.lo[k]);
        u.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
    return u;
}
__device__ __forceinline__ float half_area(const Aabb& b) {
    const float x = b.hi[0] - b.lo[0], y = b.hi[1] - b.lo[1], z = b.hi[2] - b.lo[2];
    return x * y + y * z + z * x;
}

__global__ void k_ploc_init(const Aabb* __restrict__ boxes, const uint32_t* __restrict__ vals, uint32_t n,
                            Cluster* __restrict__ c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    c[i].box = boxes[vals[i]];
    c[i].id = (int32_t)~((i << LEAF_COUNT_BITS) | 1u);
}

// nn[i] = the position j != i, |i - j| <= PLOC_RADIUS, whose union with cluster i has the smallest area.
// blockDim.x == PLOC_BLOCK; the block's clusters and their neighbours are staged in shared memory.
__global__ void __launch_bounds__(PLOC_BLOCK) k_ploc_nn(const Cluster* __restrict__ c, uint32_t m,
                                                        uint32_t* __restrict__ nn) {
    __shared__ Aabb sb[PLOC_BLOCK + 2 * PLOC_RADIUS];
    const int64_t start = (int64_t)blockIdx.x * PLOC_BLOCK - PLOC_RADIUS;
    for (int t = threadIdx.x; t < PLOC_BLOCK + 2 * PLOC_RADIUS; t += blockDim.x) {
        const int64_t g = start + t;
        if (g >= 0 && g < (int64_t)m) sb[t] = c[g].box;
    }
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * PLOC_BLOCK + threadIdx.x;
    if (i >= (int64_t)m) return;
    const Aabb a = sb[threadIdx.x + PLOC_RADIUS];
    // Candidates are ordered by (area, |i - j|, parity of min(i, j), min(i, j)).  The order is the same
    // seen from either end of a pair, so the least pair of the round is always mutual (every round
    // merges), and among equal areas adjacent pairs starting at even positions win: n identical boxes
    // pair up as (0,1)(2,3)... and halve every round instead of merging one pair at a time.
    float best = FLT_MAX;
    int64_t bj = i;
    int bdist = 1 << 30, bpar = 2;
    for (int o = -PLOC_RADIUS; o <= PLOC_RADIUS; ++o) {
        const int64_t j = i + o;
        if (o == 0 || j < 0 || j >= (int64_t)m) continue;
        const float d = half_area(unite(a, sb[threadIdx.x + PLOC_RADIUS + o]));
        const int dist = o < 0 ? -o : o;
        const int64_t lo = j < i ? j : i;
        const int par = (int)(lo & 1);
        const int64_t blo = bj < i ? bj : i;
        if (d < best || (d == best && (dist < bdist || (dist == bdist && (par < bpar || (par == bpar && lo < blo)))))) {
            best = d;
            bj = j;
            bdist = dist;
            bpar = par;
        }
    }
    nn[i] = (uint32_t)bj;
}

// keep[i]: the cluster survives the round (a merged pair survives at its lower position);
// fresh[i]: position i creates a node this round.
__global__ void k_ploc_flags(const uint32_t* __restrict__ nn, uint32_t m, uint32_t* __restrict__ keep,
                             uint32_t* __restrict__ fresh) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t j = nn[i];
    const bool mutual = j < m && j != i && nn[j] == i;
    keep[i] = !(mutual && i > j);
    fresh[i] = mutual && i < j;
}

// Writes the round's nodes (index m - 2 - rank) and the round's clusters before compaction.
__global__ void k_ploc_merge(const Cluster* __restrict__ c, const uint32_t* __restrict__ nn,
                             const uint32_t* __restrict__ fresh, const uint32_t* __restrict__ rank, uint32_t m,
                             uint32_t n, Cluster* __restrict__ out, float4* __restrict__ nodes, uint32_t* error) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (!fresh[i]) {
        out[i] = c[i];
        return;
    }
    const uint32_t j = nn[i];
    const int64_t idx = (int64_t)m - 2 - (int64_t)rank[i];
    if (j >= m || idx < 0 || idx >= (int64_t)n - 1) {
        atomicOr(error, 16u);
        out[i] = c[i];
        return;
    }
    const Cluster L = c[i], R = c[j];
    float4* np = nodes + 4 * (size_t)idx;
    np[0] = make_float4(L.box.lo[0], L.box.hi[0], L.box.lo[1], L.box.hi[1]);
    np[1] = make_float4(R.box.lo[0], R.box.hi[0], R.box.lo[1], R.box.hi[1]);
    np[2] = make_float4(L.box.lo[2], L.box.hi[2], R.box.lo[2], R.box.hi[2]);
    np[3] = make_float4(__int_as_float(L.id), __int_as_float(R.id), 0.0f, 0.0f);
    out[i].box = unite(L.box, R.box);
    out[i].id = (int32_t)idx;
}

// Depth of the deepest leaf (root = 1, as the host build counts), walking the downloaded nodes; 0 if
// the links do not form a tree over nodes [0, inner).
uint32_t tree_depth(const std::vector<float>& nodes, uint32_t inner) {
    std::vector<std::pair<int32_t, uint32_t>> stack{{0, 1u}};
    uint32_t deepest = 0, visited = 0;
    while (!stack.empty()) {
        const auto [node, depth] = stack.back();
        stack.pop_back();
        if (node < 0 || (uint32_t)node >= inner || ++visited > inner) return 0;
        for (int side = 0; side < 2; ++side) {
            int32_t c;
            std::memcpy(&c, &nodes[16 * (size_t)node + 12 + side], 4);
            if (c < 0) deepest = std::max(deepest, depth + 1);
            else stack.push_back({c, depth + 1});
        }
    }
    return visited == inner ? deepest : 0;
}

// Joins the clusters PLOC left with the host's binned SAH build (one cluster per leaf) and writes its
// k - 1 inner nodes into nodes [0, k - 2] of `nodes` (root 0), each leaf slot pointing at its cluster
// (a PLOC node or a primitive leaf).  PLOC's nearest-neighbour merges make good lower levels; a tree's
// upper levels, which every ray walks, come out better from the SAH split search.
bool join_top(const std::vector<Cluster>& rest, std::vector<float>& nodes, const char** what) {
    BvhInput tin;
    tin.boxes.resize(rest.size());
    for (size_t i = 0; i < rest.size(); ++i) tin.boxes[i] = rest[i].box;
    BvhOutput top;
    const char* terr = nullptr;
    if (!build_bvh(tin, 1, 0, top, &terr) || top.num_nodes != rest.size() - 1) {
        *what = terr ? terr : "device BVH build: the top-level join failed";
        return false;
    }
    for (uint32_t t = 0; t < top.num_nodes; ++t) {
        float* f = &top.nodes[16 * (size_t)t];
        for (int side = 0; side < 2; ++side) {
            int32_t c;
            std::memcpy(&c, &f[12 + side], 4);
            if (c < 0) {
                const uint32_t first = (uint32_t)~c >> LEAF_COUNT_BITS;
                c = rest[top.order[first]].id;
                std::memcpy(&f[12 + side], &c, 4);
            }
        }
        std::memcpy(&nodes[16 * (size_t)t], f, 16 * sizeof(float));
    }
    return true;
}

template <class T>
cudaError_t dalloc(T** p, size_t n, cudaStream_t st) {
    return cudaMallocAsync((void**)p, std::max<size_t>(n, 1) * sizeof(T), st);
}

// PLOC rounds on `st` until at most `stop_at` clusters are left (at least 1); the nodes go to `nodes`.
// A round with m clusters numbers its merges from m - 2 down, so nodes [0, m_final - 2] stay free for
// the merges that remain: with stop_at = 1 they are all made here (n - 1 records, root 0); otherwise
// the remaining clusters are copied to `rest` for the host to join.  `h_count` is page-locked host
// memory for the per-round cluster count.
cudaError_t ploc(const Aabb* d_boxes, const uint32_t* vals, uint32_t n, uint32_t stop_at, float4* d_nodes,
                 uint32_t* d_error, uint32_t* h_count, std::vector<Cluster>& rest, cudaStream_t st,
                 const char** what) {
    Cluster *cur = nullptr, *tmp = nullptr, *nxt = nullptr;
    uint32_t *nn = nullptr, *keep = nullptr, *fresh = nullptr, *rank = nullptr, *nsel = nullptr;
    void* temp = nullptr;
    size_t scan_bytes = 0, sel_bytes = 0;
    cudaError_t e = cudaSuccess;
    do {
        if ((e = dalloc(&cur, n, st)) || (e = dalloc(&tmp, n, st)) || (e = dalloc(&nxt, n, st)) ||
            (e = dalloc(&nn, n, st)) || (e = dalloc(&keep, n, st)) || (e = dalloc(&fresh, n, st)) ||
            (e = dalloc(&rank, n, st)) || (e = dalloc(&nsel, 1, st)))
            break;
        if ((e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, fresh, rank, (int)n, st))) break;
        if ((e = cub::DeviceSelect::Flagged(nullptr, sel_bytes, tmp, keep, nxt, nsel, (int)n, st))) break;
        if ((e = cudaMallocAsync(&temp, std::max<size_t>(std::max(scan_bytes, sel_bytes), 1), st))) break;
        k_ploc_init<<<(n + 255) / 256, 256, 0, st>>>(d_boxes, vals, n, cur);
        if ((e = cudaGetLastError())) break;
        uint32_t m = n;
        for (int round = 0; m > std::max(stop_at, 1u); ++round) {
            if (round >= PLOC_MAX_ROUNDS) {
                *what = "device BVH build did not converge";
                break;
            }
            const unsigned g = (m + 255) / 256;
            k_ploc_nn<<<(m + PLOC_BLOCK - 1) / PLOC_BLOCK, PLOC_BLOCK, 0, st>>>(cur, m, nn);
            k_ploc_flags<<<g, 256, 0, st>>>(nn, m, keep, fresh);
            size_t b = scan_bytes;
            if ((e = cub::DeviceScan::ExclusiveSum(temp, b, fresh, rank, (int)m, st))) break;
            k_ploc_merge<<<g, 256, 0, st>>>(cur, nn, fresh, rank, m, n, tmp, d_nodes, d_error);
            if ((e = cudaGetLastError())) break;
            b = sel_bytes;
            if ((e = cub::DeviceSelect::Flagged(temp, b, tmp, keep, nxt, nsel, (int)m, st))) break;
            if ((e = cudaMemcpyAsync(h_count, nsel, sizeof(uint32_t), cudaMemcpyDeviceToHost, st))) break;
            if ((e = cudaStreamSynchronize(st))) break;
            if (*h_count >= m || *h_count == 0) {   // every round merges at least the closest pair
                *what = "device BVH build made no progress";
                break;
            }
            m = *h_count;
            std::swap(cur, nxt);
        }
        if (e == cudaSuccess && !*what && m > 1) {
            rest.resize(m);
            if ((e = cudaMemcpyAsync(rest.data(), cur, m * sizeof(Cluster), cudaMemcpyDeviceToHost, st))) break;
            e = cudaStreamSynchronize(st);
        }
    } while (false);
    for (void* p : {(void*)cur, (void*)tmp, (void*)nxt, (void*)nn, (void*)keep, (void*)fresh, (void*)rank,
                    (void*)nsel, temp})
        if (p) cudaFreeAsync(p, st);
    return e;
}

}  // namespace

int build_bvh_device(const BvhInput& in, int device, BvhDeviceMethod method, BvhOutput& out, const char** err) {
    const size_t n = in.boxes.size();
    if (n < 2 || n >= (1u << 26)) {
        if (err) *err = "device BVH build needs 2 .. 2^26-1 primitives";
        return BVH_DEVICE_UNSUPPORTED;
    }
    // centroid bounds (one host pass over the boxes the caller already computed)
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (const Aabb& b : in.boxes)
        for (int k = 0; k < 3; ++k) {
            const float c = 0.5f * (b.lo[k] + b.hi[k]);
            lo[k] = std::min(lo[k], c);
            hi[k] = std::max(hi[k], c);
        }
    float sc[3];
    for (int k = 0; k < 3; ++k) sc[k] = hi[k] > lo[k] ? 1023.0f / (hi[k] - lo[k]) : 0.0f;

    // Own non-blocking stream and stream-ordered allocations: a build never waits for (or stalls) work
    // that other threads have in flight on the device.
    RtcDeviceScope dev(device);
    cudaError_t e = dev.error();
    cudaStream_t st = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (err) *err = cudaGetErrorString(e);
        return BVH_DEVICE_ERROR;
    }
    Aabb* d_boxes = nullptr;
    uint32_t *d_keys = nullptr, *d_keys2 = nullptr, *d_vals = nullptr, *d_vals2 = nullptr, *d_flags = nullptr,
             *d_info = nullptr;
    int32_t *d_child = nullptr, *d_pint = nullptr, *d_pleaf = nullptr;
    Aabb* d_nbox = nullptr;
    float4* d_nodes = nullptr;
    void* d_temp = nullptr;
    size_t temp_bytes = 0;
    int rc = BVH_DEVICE_ERROR;
    const char* what = nullptr;
    uint32_t* h_info = nullptr;
    std::vector<Cluster> rest;   // clusters PLOC leaves for the host's top-level join
    do {
        if ((e = dalloc(&d_boxes, n, st)) || (e = dalloc(&d_keys, n, st)) || (e = dalloc(&d_keys2, n, st)) ||
            (e = dalloc(&d_vals, n, st)) || (e = dalloc(&d_vals2, n, st)) || (e = dalloc(&d_flags, n, st)) ||
            (e = dalloc(&d_info, 4, st)) || (e = dalloc(&d_child, 2 * n, st)) || (e = dalloc(&d_pint, n, st)) ||
            (e = dalloc(&d_pleaf, n, st)) || (e = dalloc(&d_nbox, n, st)) || (e = dalloc(&d_nodes, 4 * n, st)))
            break;
        if ((e = cudaMallocHost((void**)&h_info, 4 * sizeof(uint32_t)))) break;
        if ((e = cudaMemcpyAsync(d_boxes, in.boxes.data(), n * sizeof(Aabb), cudaMemcpyHostToDevice, st))) break;
        if ((e = cudaMemsetAsync(d_flags, 0, n * sizeof(uint32_t), st))) break;
        if ((e = cudaMemsetAsync(d_child, 0xFF, 2 * n * sizeof(int32_t), st))) break;
        if ((e = cudaMemsetAsync(d_pint, 0xFF, n * sizeof(int32_t), st))) break;
        if ((e = cudaMemsetAsync(d_pleaf, 0xFF, n * sizeof(int32_t), st))) break;
        if ((e = cudaMemsetAsync(d_info, 0, 4 * sizeof(uint32_t), st))) break;
        const unsigned grid = (unsigned)((n + 255) / 256);
        k_morton<<<grid, 256, 0, st>>>(d_boxes, (uint32_t)n, make_float3(lo[0], lo[1], lo[2]),
                                       make_float3(sc[0], sc[1], sc[2]), d_keys, d_vals);
        if ((e = cudaGetLastError())) break;
        cub::DoubleBuffer<uint32_t> K(d_keys, d_keys2), V(d_vals, d_vals2);
        if ((e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, K, V, (int)n, 0, 30, st))) break;
        if ((e = cudaMallocAsync(&d_temp, std::max<size_t>(temp_bytes, 1), st))) break;
        if ((e = cub::DeviceRadixSort::SortPairs(d_temp, temp_bytes, K, V, (int)n, 0, 30, st))) break;
        const uint32_t* keys = K.Current();
        const uint32_t* vals = V.Current();
        if (method == BVH_DEVICE_LBVH) {
            k_internal<<<grid, 256, 0, st>>>(keys, (uint32_t)n, d_child, d_pint, d_pleaf, d_info);
            if ((e = cudaGetLastError())) break;
            k_bottom_up<<<grid, 256, 0, st>>>(d_boxes, vals, (uint32_t)n, d_child, d_pint, d_pleaf, d_flags, d_nbox,
                                              d_nodes, d_info + 1, d_info);
            if ((e = cudaGetLastError())) break;
        } else {
            e = ploc(d_boxes, vals, (uint32_t)n, RTC_PLOC_TOP, d_nodes, d_info, h_info + 2, rest, st, &what);
            if (e == cudaSuccess && what) rc = BVH_DEVICE_TOO_DEEP;   // no tree: the SAH build takes over
            if (e != cudaSuccess || what) break;
        }
        out.nodes.resize((n - 1) * 16);
        out.order.resize(n);
        if ((e = cudaMemcpyAsync(h_info, d_info, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st))) break;
        if ((e = cudaMemcpyAsync(out.nodes.data(), d_nodes, (n - 1) * 16 * sizeof(float), cudaMemcpyDeviceToHost, st)))
            break;
        if ((e = cudaMemcpyAsync(out.order.data(), vals, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st))) break;
        if ((e = cudaStreamSynchronize(st))) break;
        if (h_info[0]) {
            what = "device BVH build produced an inconsistent tree";
            break;
        }
        if (rest.size() > 1 && !join_top(rest, out.nodes, &what)) {
            rc = BVH_DEVICE_TOO_DEEP;   // the SAH build takes over
            break;
        }
        out.num_nodes = (uint32_t)(n - 1);
        out.max_depth = method == BVH_DEVICE_LBVH ? h_info[1] : tree_depth(out.nodes, (uint32_t)(n - 1));
        if (out.max_depth == 0) {
            what = "device BVH build produced an inconsistent tree";
            break;
        }
        out.max_leaf_seen = 1;
        out.nodes8.clear();
        out.items8.clear();
        out.num_nodes8 = 0;
        // one primitive per leaf so far: with RTC_DEVICE_LEAF_MAX > 1, merge small subtrees into leaves of
        // up to that many where the SAH cost favours it, as the host build's leaves are
        if (RTC_DEVICE_LEAF_MAX > 1) collapse_leaves(out, RTC_DEVICE_LEAF_MAX);
        if (out.max_depth + 2 > (uint32_t)TRAVERSAL_STACK) {
            what = "device BVH too deep for the traversal stack";
            rc = BVH_DEVICE_TOO_DEEP;
        } else {
            rc = BVH_DEVICE_OK;
        }
    } while (false);
    for (void* p : {(void*)d_boxes, (void*)d_keys, (void*)d_keys2, (void*)d_vals, (void*)d_vals2, (void*)d_flags,
                    (void*)d_info, (void*)d_child, (void*)d_pint, (void*)d_pleaf, (void*)d_nbox, (void*)d_nodes, d_temp})
        if (p) cudaFreeAsync(p, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (h_info) cudaFreeHost(h_info);
    cudaStreamDestroy(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) rc = BVH_DEVICE_ERROR;
    if (rc != BVH_DEVICE_OK && err) *err = e != cudaSuccess ? cudaGetErrorString(e) : what;
    return rc;
}

}  // namespace rtc
