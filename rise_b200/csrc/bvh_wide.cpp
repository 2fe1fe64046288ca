// bvh_wide.cpp -- the 8-wide compressed device layout (WNode8).
//
// The reference's BVH2 (the same tree the other layouts collapse to four-wide
// nodes) is collapsed here to eight-wide nodes of 80 bytes, after the
// compressed wide BVH of Ylitie, Karras and Laine ("Efficient Incoherent Ray
// Traversal on GPUs Through Compressed Wide BVHs", HPG 2017):
//  * a node's children are gathered by repeatedly opening the largest-area
//    internal child while the slots allow; a leaf takes one slot per three
//    triangles (the reference's leaves hold at most four, so two at most);
//  * children sit in slots by octant: slot s is meant for the child lying
//    furthest along the direction whose component k is -1 where bit k of s
//    is set, +1 elsewhere (greedy assignment by centroid offset from the
//    node's centre), so a ray that visits slots in the order s ^ x, x the
//    bits of its non-negative direction components, meets children roughly
//    near to far without sorting;
//  * child boxes are 8-bit bounds against a per-node origin and power-of-two
//    scale per axis, rounded outward and checked to contain the FP32 boxes,
//    so culling is conservative and the FP32 watertight triangle test decides
//    every hit;
//  * internal children are stored contiguously (breadth-first), a leaf
//    slot's triangles contiguously from the node's triangle base; a leaf
//    slot's meta byte holds its triangle count in unary above a 5-bit offset,
//    so one shift per slot builds the node's triangle hit mask.
// Hit ids do not depend on the tree shape (except at exact distance ties,
// which the parity rules count), so the reference's hits are kept.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "bvh_build.h"

namespace rtb200 {

namespace {

struct Box {
    float lo[3], hi[3];
};

float Area(const Box& b)
{
    const double dx = (double)b.hi[0] - b.lo[0], dy = (double)b.hi[1] - b.lo[1], dz = (double)b.hi[2] - b.lo[2];
    return (float)(dx * dy + dy * dz + dz * dx);
}

// One slot of a node under construction: an internal BVH2 node, or a run of
// at most three triangles of a BVH2 leaf (leaf-order slots first..first+count).
struct Slot {
    bool internal;
    uint32_t node2;      // internal: BVH2 node index
    uint32_t first;      // leaf run: first leaf-order prim slot
    uint32_t count;
    Box box;
};

Box NodeBox(const Node2& n)
{
    Box b;
    for (int k = 0; k < 3; ++k) { b.lo[k] = n.bmin[k]; b.hi[k] = n.bmax[k]; }
    return b;
}

int SlotsOf(const Node2& n) { return n.count > 0 ? (int)((n.count + 2) / 3) : 1; }

inline float DecodeQ(float o, int e, int q) { return o + (float)q * std::ldexp(1.0f, e); }

}  // namespace

bool EncodeWideNodes(const BuiltBVH& b, std::vector<WNode8>& nodes, std::vector<uint32_t>& prims, int& depth)
{
    nodes.clear();
    prims.clear();
    depth = 0;
    const std::vector<Node2>& n2 = b.nodes2;
    if (n2.empty()) return true;
    // The node queue: BVH2 nodes that head a wide node, in breadth-first
    // order, with their wide-tree level.
    std::vector<std::pair<uint32_t, int>> queue{{0u, 1}};
    for (size_t head = 0; head < queue.size(); ++head) {
        const uint32_t root2 = queue[head].first;
        const int level = queue[head].second;
        depth = std::max(depth, level);
        // Gather children: start from this BVH2 node's two children (or the
        // node itself when it is a leaf, which only a one-leaf tree's root is).
        std::vector<uint32_t> kids;
        if (n2[root2].count > 0) {
            kids.push_back(root2);
        } else {
            kids.push_back(n2[root2].first_or_left);
            kids.push_back(n2[root2].first_or_left + 1);
        }
        auto total = [&]() {
            int t = 0;
            for (uint32_t k : kids) t += SlotsOf(n2[k]);
            return t;
        };
        if (total() > 8) return false;   // a leaf of more than 24 triangles
        for (;;) {
            int best = -1;
            float bestArea = -1.0f;
            const int t = total();
            for (size_t i = 0; i < kids.size(); ++i) {
                const Node2& c = n2[kids[i]];
                if (c.count > 0) continue;
                const int grow = SlotsOf(n2[c.first_or_left]) + SlotsOf(n2[c.first_or_left + 1]) - 1;
                if (t + grow > 8) continue;
                const float a = Area(NodeBox(c));
                if (a > bestArea) { bestArea = a; best = (int)i; }
            }
            if (best < 0) break;
            const uint32_t c = kids[best];
            kids[best] = n2[c].first_or_left;
            kids.push_back(n2[c].first_or_left + 1);
        }
        std::vector<Slot> slots;
        for (uint32_t k : kids) {
            const Node2& c = n2[k];
            if (c.count == 0) {
                slots.push_back({true, k, 0, 0, NodeBox(c)});
            } else {
                for (uint32_t off = 0; off < c.count; off += 3)
                    slots.push_back({false, 0, c.first_or_left + off, std::min<uint32_t>(3, c.count - off), NodeBox(c)});
            }
        }
        // Octant slots: child i into slot s maximising its centroid offset
        // along direction s (greedy over the pairs, largest first).
        Box u{{FLT_MAX, FLT_MAX, FLT_MAX}, {-FLT_MAX, -FLT_MAX, -FLT_MAX}};
        for (const Slot& s : slots)
            for (int k = 0; k < 3; ++k) { u.lo[k] = std::min(u.lo[k], s.box.lo[k]); u.hi[k] = std::max(u.hi[k], s.box.hi[k]); }
        struct Pair { float cost; int child, slot; };
        std::vector<Pair> pairs;
        for (int i = 0; i < (int)slots.size(); ++i)
            for (int sl = 0; sl < 8; ++sl) {
                float c = 0.0f;
                for (int k = 0; k < 3; ++k) {
                    const float off = 0.5f * ((slots[i].box.lo[k] + slots[i].box.hi[k]) - (u.lo[k] + u.hi[k]));
                    c += ((sl >> k) & 1) ? -off : off;
                }
                pairs.push_back({c, i, sl});
            }
        std::stable_sort(pairs.begin(), pairs.end(), [](const Pair& a, const Pair& b2) { return a.cost > b2.cost; });
        int at[8];
        std::fill(at, at + 8, -1);
        std::vector<bool> placed(slots.size(), false);
        for (const Pair& p : pairs) {
            if (placed[p.child] || at[p.slot] >= 0) continue;
            at[p.slot] = p.child;
            placed[p.child] = true;
        }
        // Encode.
        WNode8 d;
        std::memset(&d, 0, sizeof(d));
        float org[3];
        int ex[3];
        for (int k = 0; k < 3; ++k) {
            org[k] = u.lo[k];
            const double ext = (double)u.hi[k] - (double)u.lo[k];
            int e = -126;
            if (ext > 0) {
                e = (int)std::ceil(std::log2(ext / 254.0));
                while (254.0 * std::ldexp(1.0, e) < ext) ++e;
                if (e < -126) e = -126;
            }
            ex[k] = e;
        }
        d.px = org[0]; d.py = org[1]; d.pz = org[2];
        d.ex = (int8_t)ex[0]; d.ey = (int8_t)ex[1]; d.ez = (int8_t)ex[2];
        d.child_base = (uint32_t)queue.size();
        d.tri_base = (uint32_t)prims.size();
        uint8_t* qlo[3] = {d.qlox, d.qloy, d.qloz};
        uint8_t* qhi[3] = {d.qhix, d.qhiy, d.qhiz};
        uint32_t tri_off = 0;
        for (int sl = 0; sl < 8; ++sl) {
            const int i = at[sl];
            if (i < 0) {
                for (int k = 0; k < 3; ++k) { qlo[k][sl] = 255; qhi[k][sl] = 0; }
                continue;
            }
            const Slot& s = slots[i];
            for (int k = 0; k < 3; ++k) {
                const double sc = std::ldexp(1.0, ex[k]);
                int ql = (int)std::floor(((double)s.box.lo[k] - org[k]) / sc);
                int qh = (int)std::ceil(((double)s.box.hi[k] - org[k]) / sc);
                ql = std::max(0, std::min(255, ql));
                qh = std::max(0, std::min(255, qh));
                while (ql > 0 && DecodeQ(org[k], ex[k], ql) >= s.box.lo[k]) --ql;
                while (qh < 255 && DecodeQ(org[k], ex[k], qh) <= s.box.hi[k]) ++qh;
                qlo[k][sl] = (uint8_t)ql;
                qhi[k][sl] = (uint8_t)qh;
            }
            if (s.internal) {
                d.imask |= (uint8_t)(1u << sl);
                queue.push_back({s.node2, level + 1});
            } else {
                d.meta[sl] = (uint8_t)((((1u << s.count) - 1u) << 5) | tri_off);
                for (uint32_t t = 0; t < s.count; ++t) prims.push_back(b.prims[s.first + t]);
                tri_off += s.count;
            }
        }
        nodes.push_back(d);
    }
    return true;
}

void EncodeWideTriangles(const float* tri9, const std::vector<uint32_t>& prims, std::vector<GpuTri>& out)
{
    out.resize(prims.size());
    for (size_t i = 0; i < prims.size(); ++i) {
        const uint32_t p = prims[i];
        const float* s = tri9 + 9 * (size_t)p;
        GpuTri& t = out[i];
        for (int k = 0; k < 3; ++k) { t.v0[k] = s[k]; t.v1[k] = s[3 + k]; t.v2[k] = s[6 + k]; }
        std::memcpy(&t.v0[3], &p, 4);
        t.v1[3] = 1.0f;   // every triangle is its own run: no leaf walk continues past it
        t.v2[3] = 0.0f;
    }
}

}  // namespace rtb200
