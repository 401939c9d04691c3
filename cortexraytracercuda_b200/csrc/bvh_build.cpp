// bvh_build.cpp - binned SAH BVH2 builder (host).  See bvh_build.h.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <tuple>

#include "rtc_dev.h"

namespace rtc {
namespace {

constexpr int NBINS = 32;
constexpr int MAX_TREE_DEPTH = 56;   // < TRAVERSAL_STACK, leaves room for the root pair

struct BNode {
    Aabb box;
    int32_t left = -1, right = -1;   // children (node ids) for inner nodes
    uint32_t first = 0, count = 0;   // leaf range in the index array
    bool leaf = false;
};

inline void grow(Aabb& a, const Aabb& b) {
    for (int k = 0; k < 3; ++k) {
        a.lo[k] = std::min(a.lo[k], b.lo[k]);
        a.hi[k] = std::max(a.hi[k], b.hi[k]);
    }
}
inline Aabb empty_box() {
    Aabb a;
    for (int k = 0; k < 3; ++k) { a.lo[k] = FLT_MAX; a.hi[k] = -FLT_MAX; }
    return a;
}
inline double area(const Aabb& a) {
    double dx = (double)a.hi[0] - a.lo[0], dy = (double)a.hi[1] - a.lo[1], dz = (double)a.hi[2] - a.lo[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.0;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

constexpr int PAR_DEPTH = 4;            // subtrees below the first four levels are built concurrently
constexpr uint32_t PAR_MIN = 32768;     // ... when they hold at least this many primitives

struct Shared {
    const std::vector<Aabb>& boxes;
    std::vector<float> cen;          // 3 per primitive
    std::vector<uint32_t> idx;       // subtrees partition disjoint ranges of it
    int max_leaf;
};

struct Builder {
    Shared& sh;
    const std::vector<Aabb>& boxes;
    std::vector<float>& cen;
    std::vector<uint32_t>& idx;
    int max_leaf;
    std::vector<BNode> nodes;        // per-builder (one per subtree task)

    explicit Builder(Shared& s) : sh(s), boxes(s.boxes), cen(s.cen), idx(s.idx), max_leaf(s.max_leaf) {}

    // Appends another builder's tree (its node 0 is its root); returns the root's id here.
    int32_t splice(const Builder& o) {
        const int32_t off = (int32_t)nodes.size();
        for (BNode b : o.nodes) {
            if (!b.leaf) {
                b.left += off;
                b.right += off;
            }
            nodes.push_back(b);
        }
        return off;
    }

    int32_t build(uint32_t start, uint32_t end, int depth, uint32_t& max_depth) {
        int32_t id = (int32_t)nodes.size();
        nodes.emplace_back();
        Aabb box = empty_box(), cb = empty_box();
        for (uint32_t i = start; i < end; ++i) {
            uint32_t p = idx[i];
            grow(box, boxes[p]);
            for (int k = 0; k < 3; ++k) {
                cb.lo[k] = std::min(cb.lo[k], cen[3 * p + k]);
                cb.hi[k] = std::max(cb.hi[k], cen[3 * p + k]);
            }
        }
        nodes[id].box = box;
        if ((uint32_t)depth > max_depth) max_depth = depth;
        const uint32_t n = end - start;
        auto make_leaf = [&]() {
            nodes[id].leaf = true;
            nodes[id].first = start;
            nodes[id].count = n;
            return id;
        };
        if (n <= 1) return make_leaf();

        // best binned SAH split
        int best_axis = -1, best_bin = -1;
        double best_cost = DBL_MAX;
        const double parea = std::max(area(box), 1e-30);
        for (int ax = 0; ax < 3; ++ax) {
            double ext = (double)cb.hi[ax] - cb.lo[ax];
            if (!(ext > 0.0)) continue;
            uint32_t cnt[NBINS] = {0};
            Aabb bb[NBINS];
            for (int b = 0; b < NBINS; ++b) bb[b] = empty_box();
            const double scale = NBINS / ext;
            for (uint32_t i = start; i < end; ++i) {
                uint32_t p = idx[i];
                int b = (int)(((double)cen[3 * p + ax] - cb.lo[ax]) * scale);
                b = b < 0 ? 0 : (b >= NBINS ? NBINS - 1 : b);
                cnt[b]++;
                grow(bb[b], boxes[p]);
            }
            double la[NBINS];
            uint32_t lc[NBINS];
            Aabb acc = empty_box();
            uint32_t c = 0;
            for (int b = 0; b < NBINS - 1; ++b) {
                grow(acc, bb[b]);
                c += cnt[b];
                la[b] = area(acc);
                lc[b] = c;
            }
            acc = empty_box();
            c = 0;
            for (int b = NBINS - 1; b > 0; --b) {
                grow(acc, bb[b]);
                c += cnt[b];
                uint32_t nl = lc[b - 1];
                if (nl == 0 || c == 0) continue;
                double cost = 1.0 + (la[b - 1] * nl + area(acc) * c) / parea;
                if (cost < best_cost) { best_cost = cost; best_axis = ax; best_bin = b; }
            }
        }
        const bool can_leaf = n <= (uint32_t)max_leaf;
        if (can_leaf && (best_axis < 0 || (double)n <= best_cost)) return make_leaf();

        uint32_t mid;
        if (best_axis >= 0 && depth < MAX_TREE_DEPTH) {
            const double ext = (double)cb.hi[best_axis] - cb.lo[best_axis];
            const double scale = NBINS / ext;
            auto it = std::partition(idx.begin() + start, idx.begin() + end, [&](uint32_t p) {
                int b = (int)(((double)cen[3 * p + best_axis] - cb.lo[best_axis]) * scale);
                b = b < 0 ? 0 : (b >= NBINS ? NBINS - 1 : b);
                return b < best_bin;
            });
            mid = (uint32_t)(it - idx.begin());
            if (mid == start || mid == end) mid = start + n / 2;
        } else {
            // median split on the widest centroid axis (also the fallback for coincident centroids)
            int ax = 0;
            for (int k = 1; k < 3; ++k)
                if (cb.hi[k] - cb.lo[k] > cb.hi[ax] - cb.lo[ax]) ax = k;
            mid = start + n / 2;
            std::nth_element(idx.begin() + start, idx.begin() + mid, idx.begin() + end,
                             [&](uint32_t a, uint32_t b) { return cen[3 * a + ax] < cen[3 * b + ax]; });
        }
        if (depth <= PAR_DEPTH && n >= PAR_MIN) {
            // the two halves on two threads, each into its own node array, then spliced in
            Builder L(sh), R(sh);
            uint32_t dl = 0, dr = 0;
            std::thread t([&] { L.build(start, mid, depth + 1, dl); });
            R.build(mid, end, depth + 1, dr);
            t.join();
            max_depth = std::max(max_depth, std::max(dl, dr));
            const int32_t l = splice(L);
            const int32_t r = splice(R);
            nodes[id].left = l;
            nodes[id].right = r;
            return id;
        }
        int32_t l = build(start, mid, depth + 1, max_depth);
        int32_t r = build(mid, end, depth + 1, max_depth);
        nodes[id].left = l;
        nodes[id].right = r;
        return id;
    }
};

}  // namespace

bool build_bvh(const BvhInput& in, int max_leaf, int threads, BvhOutput& out, const char** err) {
    (void)threads;
    const size_t n = in.boxes.size();
    if (max_leaf < 1) max_leaf = 1;
    if (max_leaf > MAX_LEAF) max_leaf = MAX_LEAF;
    if (n >= (1u << 26)) { if (err) *err = "too many primitives for the leaf encoding (max 2^26)"; return false; }
    Shared SH{in.boxes, {}, {}, max_leaf};
    SH.cen.resize(3 * n);
    SH.idx.resize(n);
    for (size_t p = 0; p < n; ++p) {
        SH.idx[p] = (uint32_t)p;
        for (int k = 0; k < 3; ++k) SH.cen[3 * p + k] = 0.5f * (in.boxes[p].lo[k] + in.boxes[p].hi[k]);
    }
    Builder B(SH);
    B.nodes.reserve(2 * n + 2);
    uint32_t max_depth = 0;
    int32_t root = n ? B.build(0, (uint32_t)n, 1, max_depth) : -1;

    // Flatten: inner nodes in depth-first order, leaves folded into their parent's child slots.
    out.nodes.clear();
    out.order.clear();
    out.max_leaf_seen = 0;
    std::vector<int32_t> stack;
    auto alloc_node = [&]() {
        out.nodes.resize(out.nodes.size() + 16, 0.0f);
        return (int32_t)(out.nodes.size() / 16 - 1);
    };
    auto encode_leaf = [&](const BNode& L) -> int32_t {
        uint32_t first = (uint32_t)out.order.size();
        for (uint32_t i = 0; i < L.count; ++i) out.order.push_back(B.idx[L.first + i]);
        if (L.count > out.max_leaf_seen) out.max_leaf_seen = L.count;
        return (int32_t)~((first << LEAF_COUNT_BITS) | L.count);
    };
    auto put_child = [&](int32_t slot, int side, const Aabb& bx, int32_t enc) {
        float* f = &out.nodes[16 * (size_t)slot];
        if (side == 0) {
            f[0] = bx.lo[0]; f[1] = bx.hi[0]; f[2] = bx.lo[1]; f[3] = bx.hi[1];
            f[8] = bx.lo[2]; f[9] = bx.hi[2];
            std::memcpy(&f[12], &enc, 4);
        } else {
            f[4] = bx.lo[0]; f[5] = bx.hi[0]; f[6] = bx.lo[1]; f[7] = bx.hi[1];
            f[10] = bx.lo[2]; f[11] = bx.hi[2];
            std::memcpy(&f[13], &enc, 4);
        }
    };
    // root slot 0: if the whole tree is one leaf, pair it with an empty leaf
    struct Pending { int32_t bnode; int32_t slot; int side; };
    std::vector<Pending> work;
    int32_t slot0 = alloc_node();
    Aabb none = empty_box();
    if (root < 0) {
        put_child(slot0, 0, none, (int32_t)~0u);
        put_child(slot0, 1, none, (int32_t)~0u);
    } else if (B.nodes[root].leaf) {
        put_child(slot0, 0, B.nodes[root].box, encode_leaf(B.nodes[root]));
        put_child(slot0, 1, none, (int32_t)~0u);
    } else {
        work.push_back({B.nodes[root].right, slot0, 1});
        work.push_back({B.nodes[root].left, slot0, 0});
        while (!work.empty()) {
            Pending w = work.back();
            work.pop_back();
            const BNode& bn = B.nodes[w.bnode];
            if (bn.leaf) {
                put_child(w.slot, w.side, bn.box, encode_leaf(bn));
            } else {
                int32_t s = alloc_node();
                put_child(w.slot, w.side, bn.box, s);
                work.push_back({bn.right, s, 1});
                work.push_back({bn.left, s, 0});
            }
        }
    }
    out.num_nodes = (uint32_t)(out.nodes.size() / 16);
    out.max_depth = max_depth;

    // 8-wide collapse of the same tree: quantised child boxes, slots in octant order, links by base
    // index (the compressed wide layout of Ylitie, Karras and Laine, HPG 2017, restated for this
    // tree's leaves).
    //  * Children: a wide node starts with its binary node's two children and repeatedly opens the
    //    inner child of largest surface area, up to eight.
    //  * Slots: bit k of slot s means the high side of axis k.  Each child goes to the slot whose
    //    diagonal direction (+-1, +-1, +-1) best matches the offset of its box centre from the node's
    //    (greedy assignment, largest dot product first).  A ray whose direction has sign bits `oct`
    //    visits slot j ^ oct at step j: the child at the corner the ray enters from comes first.
    //  * Links: inner children get consecutive node indices in slot order (node = base + rank).  Leaf
    //    children's item ranges are copied, in slot order, to consecutive entries of a second item
    //    list (`items8`, entries = positions in `order`), so a leaf is (item base + offset, count).
    //    One byte per slot: 0x80 | rank for an inner child, (count - 1) << 5 | offset for a leaf; the
    //    node's valid mask marks the slots in use.
    //  * Boxes: the node's low corner p, one power-of-two step 2^e per axis with 255 * 2^e >= the
    //    box's extent, and per child and axis 8-bit bounds floor((lo - p) / 2^e) and
    //    ceil((hi - p) / 2^e): p + q * 2^e encloses the child's box (checked in double below), so the
    //    quantised test never loses a hit the binary nodes find.
    out.nodes8.clear();
    out.items8.clear();
    auto alloc8 = [&](int count) {
        const int32_t first = (int32_t)(out.nodes8.size() / NODE8_FLOATS);
        out.nodes8.resize(out.nodes8.size() + (size_t)count * NODE8_FLOATS, 0.0f);
        return first;
    };
    // the binary flattening's leaf encoding of each binary leaf (replayed in its DFS left-first order)
    std::vector<int32_t> leaf_of(B.nodes.size(), 0);
    {
        std::vector<int32_t> st;
        if (root >= 0) st.push_back(root);
        uint32_t first = 0;
        while (!st.empty()) {
            int32_t b = st.back();
            st.pop_back();
            const BNode& bn = B.nodes[b];
            if (bn.leaf) {
                leaf_of[b] = (int32_t)~((first << LEAF_COUNT_BITS) | bn.count);
                first += bn.count;
            } else {
                st.push_back(bn.right);
                st.push_back(bn.left);
            }
        }
    }
    struct Work8 { int32_t bnode; int32_t slot; uint32_t depth; };
    bool wide_ok = true;
    // writes wide node `at` from `n` children (binary node ids); inner children are queued on `kids`
    auto put8 = [&](int32_t at, const int32_t* ch, int n, uint32_t depth, std::vector<Work8>& kids) {
        Aabb nb;
        for (int k = 0; k < 3; ++k) { nb.lo[k] = INFINITY; nb.hi[k] = -INFINITY; }
        for (int i = 0; i < n; ++i) grow(nb, B.nodes[ch[i]].box);
        // slot assignment
        double score[8][8];
        for (int i = 0; i < n; ++i) {
            const Aabb& c = B.nodes[ch[i]].box;
            double off[3];
            for (int k = 0; k < 3; ++k)
                off[k] = 0.5 * ((double)c.lo[k] + (double)c.hi[k]) - 0.5 * ((double)nb.lo[k] + (double)nb.hi[k]);
            for (int sl = 0; sl < 8; ++sl)
                score[i][sl] = ((sl & 1) ? off[0] : -off[0]) + ((sl & 2) ? off[1] : -off[1]) +
                               ((sl & 4) ? off[2] : -off[2]);
        }
        int child_in[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        bool placed[8] = {};
        for (int round = 0; round < n; ++round) {
            int bi = -1, bs = -1;
            double best = -INFINITY;
            for (int i = 0; i < n; ++i) {
                if (placed[i]) continue;
                for (int sl = 0; sl < 8; ++sl)
                    if (child_in[sl] < 0 && score[i][sl] > best) { best = score[i][sl]; bi = i; bs = sl; }
            }
            placed[bi] = true;
            child_in[bs] = bi;
        }
        // links
        int inner = 0;
        for (int sl = 0; sl < 8; ++sl)
            if (child_in[sl] >= 0 && !B.nodes[ch[child_in[sl]]].leaf) ++inner;
        const int32_t base = inner ? alloc8(inner) : 0;
        const uint32_t item_base = (uint32_t)out.items8.size();
        uint32_t valid = 0, meta[2] = {0u, 0u};
        int rank = 0;
        for (int sl = 0; sl < 8; ++sl) {
            if (child_in[sl] < 0) continue;
            const int32_t b = ch[child_in[sl]];
            valid |= 1u << sl;
            uint32_t byte;
            if (B.nodes[b].leaf) {
                const uint32_t enc = (uint32_t)~leaf_of[b];
                const uint32_t first = enc >> LEAF_COUNT_BITS, cnt = enc & MAX_LEAF;
                const uint32_t off = (uint32_t)out.items8.size() - item_base;
                if (cnt < 1 || cnt > 4 || off > 31) wide_ok = false;
                byte = ((cnt - 1u) & 3u) << 5 | (off & 31u);
                for (uint32_t i = 0; i < cnt; ++i) out.items8.push_back(first + i);
            } else {
                byte = 0x80u | (uint32_t)rank;
                kids.push_back({b, base + rank, depth + 1});
                ++rank;
            }
            meta[sl >> 2] |= byte << (8 * (sl & 3));
        }
        // quantised boxes
        uint32_t hdr = valid << 24;
        uint8_t q[3][2][8] = {};   // axis, (low, high), slot
        for (int k = 0; k < 3; ++k) {
            const double ext = (double)nb.hi[k] - (double)nb.lo[k];
            int e = -126;
            while (e < 127 && std::ldexp(255.0, e) < ext) ++e;
            const double step = std::ldexp(1.0, e);
            hdr |= (uint32_t)(e + 127) << (8 * k);
            for (int sl = 0; sl < 8; ++sl) {
                if (child_in[sl] < 0) continue;
                const Aabb& c = B.nodes[ch[child_in[sl]]].box;
                const double ql = std::floor(((double)c.lo[k] - (double)nb.lo[k]) / step);
                const double qh = std::ceil(((double)c.hi[k] - (double)nb.lo[k]) / step);
                const double l = std::min(std::max(ql, 0.0), 255.0), h = std::min(std::max(qh, 0.0), 255.0);
                if ((double)nb.lo[k] + l * step > (double)c.lo[k] || (double)nb.lo[k] + h * step < (double)c.hi[k])
                    wide_ok = false;
                q[k][0][sl] = (uint8_t)l;
                q[k][1][sl] = (uint8_t)h;
            }
        }
        float* f = &out.nodes8[NODE8_FLOATS * (size_t)at];   // after alloc8: nodes8 may have moved
        f[0] = nb.lo[0];
        f[1] = nb.lo[1];
        f[2] = nb.lo[2];
        std::memcpy(&f[3], &hdr, 4);
        std::memcpy(&f[4], &base, 4);
        std::memcpy(&f[5], &item_base, 4);
        std::memcpy(&f[6], &meta[0], 4);
        std::memcpy(&f[7], &meta[1], 4);
        for (int k = 0; k < 3; ++k) {   // float4 2 + k: low bytes of slots 0-7, then high bytes
            std::memcpy(&f[8 + 4 * k], q[k][0], 8);
            std::memcpy(&f[10 + 4 * k], q[k][1], 8);
        }
    };
    std::vector<Work8> w8, kids;
    uint32_t depth8 = 1;
    const int32_t r8 = alloc8(1);
    if (root >= 0) {
        if (B.nodes[root].leaf) {
            put8(r8, &root, 1, 1, kids);
        } else {
            w8.push_back({root, r8, 1});
        }
    }
    while (!w8.empty()) {
        Work8 w = w8.back();
        w8.pop_back();
        depth8 = std::max(depth8, w.depth);
        const BNode& bn = B.nodes[w.bnode];
        int32_t ch[8] = {bn.left, bn.right, -1, -1, -1, -1, -1, -1};
        int n = 2;
        while (n < 8) {
            int best = -1;
            double ba = -1.0;
            for (int i = 0; i < n; ++i) {
                const BNode& c = B.nodes[ch[i]];
                if (!c.leaf && area(c.box) > ba) { ba = area(c.box); best = i; }
            }
            if (best < 0) break;
            const BNode& o = B.nodes[ch[best]];
            for (int i = n; i > best + 1; --i) ch[i] = ch[i - 1];
            ch[best] = o.left;
            ch[best + 1] = o.right;
            ++n;
        }
        kids.clear();
        put8(w.slot, ch, n, w.depth, kids);
        // depth first, first slot next: a node's subtree sits close to it in memory
        for (auto it = kids.rbegin(); it != kids.rend(); ++it) w8.push_back(*it);
    }
    out.num_nodes8 = (uint32_t)(out.nodes8.size() / NODE8_FLOATS);
    // the walk keeps at most one pending group per level; nodes are addressed with 24 bits on its stack
    if (!wide_ok || depth8 + 1 > (uint32_t)TRAVERSAL_STACK8 || out.num_nodes8 >= (1u << 24)) {
        out.nodes8.clear();   // renders use the binary nodes
        out.items8.clear();
        out.num_nodes8 = 0;
    }
    if (max_depth + 2 > (uint32_t)TRAVERSAL_STACK) { if (err) *err = "BVH too deep for the traversal stack"; return false; }
    return true;
}

// Collapses subtrees of at most `max_leaf` primitives into leaves where the SAH cost says a leaf is
// cheaper (the host build's costs: 1 per node visit, 1 per primitive test, children weighted by their
// box's area over the parent's), renumbering the nodes in depth-first order and the leaf slots so that
// each new leaf's primitives are contiguous.  The root stays an inner node.  For trees built one
// primitive per leaf (the device builds).
void collapse_leaves(BvhOutput& t, int max_leaf) {
    const uint32_t inner = t.num_nodes;
    if (inner == 0) return;
    auto link = [&](uint32_t node, int side) {
        int32_t c;
        std::memcpy(&c, &t.nodes[16 * (size_t)node + 12 + side], 4);
        return c;
    };
    // a child's box and area, from its parent's record (L: x in [0,1], y in [2,3], z in [8,9]; R: 4-7, 10-11)
    auto child_area = [&](uint32_t node, int side) {
        const float* n = &t.nodes[16 * (size_t)node];
        const float dx = side ? n[5] - n[4] : n[1] - n[0];
        const float dy = side ? n[7] - n[6] : n[3] - n[2];
        const float dz = side ? n[11] - n[10] : n[9] - n[8];
        return 2.0 * ((double)dx * dy + (double)dy * dz + (double)dz * dx);
    };
    auto node_area = [&](uint32_t node) {
        const float* n = &t.nodes[16 * (size_t)node];
        const float dx = std::max(n[1], n[5]) - std::min(n[0], n[4]);
        const float dy = std::max(n[3], n[7]) - std::min(n[2], n[6]);
        const float dz = std::max(n[9], n[11]) - std::min(n[8], n[10]);
        return 2.0 * ((double)dx * dy + (double)dy * dz + (double)dz * dx);
    };
    std::vector<uint32_t> count(inner, 0);
    std::vector<double> cost(inner, 0.0);
    std::vector<uint8_t> leaf(inner, 0);
    // post-order over the inner nodes (explicit stack: device trees can be deep)
    std::vector<std::pair<uint32_t, bool>> st{{0u, false}};
    while (!st.empty()) {
        auto [node, done] = st.back();
        st.pop_back();
        if (!done) {
            st.push_back({node, true});
            for (int side = 0; side < 2; ++side)
                if (link(node, side) >= 0) st.push_back({(uint32_t)link(node, side), false});
            continue;
        }
        uint32_t n = 0;
        double split = 1.0;
        const double a = std::max(node_area(node), 1e-30);
        for (int side = 0; side < 2; ++side) {
            const int32_t c = link(node, side);
            const uint32_t cn = c < 0 ? ((uint32_t)~c & 31u) : count[c];
            const double cc = c < 0 ? (double)cn : cost[c];
            n += cn;
            split += child_area(node, side) * cc / a;
        }
        count[node] = n;
        leaf[node] = node != 0 && (int)n <= max_leaf && (double)n <= split;
        cost[node] = leaf[node] ? (double)n : split;
    }
    // depth-first renumbering; collapsed subtrees become leaves of contiguous slots
    std::vector<float> nodes;
    std::vector<uint32_t> order;
    nodes.reserve(t.nodes.size());
    order.reserve(t.order.size());
    uint32_t max_depth = 0, max_leaf_seen = 0;
    auto gather = [&](int32_t c) {   // appends the primitives under link c to `order`
        std::vector<int32_t> s{c};
        while (!s.empty()) {
            const int32_t x = s.back();
            s.pop_back();
            if (x < 0) {
                const uint32_t first = (uint32_t)~x >> 5, cnt = (uint32_t)~x & 31u;
                for (uint32_t k = 0; k < cnt; ++k) order.push_back(t.order[first + k]);
            } else {
                s.push_back(link((uint32_t)x, 1));
                s.push_back(link((uint32_t)x, 0));
            }
        }
    };
    // (old node, depth, where its new index goes: a link slot in `nodes`, or -1 for the root)
    std::vector<std::tuple<uint32_t, uint32_t, int64_t>> work{{0u, 1u, -1}};
    while (!work.empty()) {
        const auto [old, depth, slot] = work.back();
        work.pop_back();
        const uint32_t me = (uint32_t)(nodes.size() / 16);
        if (slot >= 0) std::memcpy(&nodes[(size_t)slot], &me, 4);
        nodes.insert(nodes.end(), t.nodes.begin() + 16 * (size_t)old, t.nodes.begin() + 16 * (size_t)old + 16);
        for (int side = 1; side >= 0; --side) {
            const int32_t c = link(old, side);
            const size_t at = 16 * (size_t)me + 12 + side;
            if (c >= 0 && !leaf[c]) {
                work.push_back({(uint32_t)c, depth + 1, (int64_t)at});
                continue;
            }
            const uint32_t first = (uint32_t)order.size();
            gather(c);
            const uint32_t cnt = (uint32_t)order.size() - first;
            const int32_t enc = ~(int32_t)((first << 5) | cnt);
            std::memcpy(&nodes[at], &enc, 4);
            max_depth = std::max(max_depth, depth + 1);
            max_leaf_seen = std::max(max_leaf_seen, cnt);
        }
    }
    t.nodes.swap(nodes);
    t.order.swap(order);
    t.num_nodes = (uint32_t)(t.nodes.size() / 16);
    t.max_depth = max_depth;
    t.max_leaf_seen = max_leaf_seen;
}

}  // namespace rtc
