// bvh_build.cpp -- see bvh_build.h.
//
// The split search follows the reference builder step for step
// (src/Library/Acceleration/BVH.h:860-1034): tight box over the range's
// primitive boxes, longest centroid-box axis, 32 uniform centroid bins, prefix
// and suffix sweeps that skip empty bins, SAH cost 1 + (A_l*N_l + A_r*N_r)/A,
// in-place partition by `centroid < splitVal` with the same swap sequence, and
// the median fallback through std::nth_element.  Doing the same double-precision
// arithmetic in the same order is what makes the trees identical.
//
// Differences from the reference are in execution only: primitive boxes and
// centroids are kept in flat arrays, subtrees above a size threshold are built
// on worker threads, and a final depth-first pass assigns node indices in the
// reference's allocation order (children of a node are allocated as an adjacent
// pair, left subtree fully numbered before the right).
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <mutex>
#include <thread>

namespace rtb200 {
namespace {

const double kInf = DBL_MAX;

struct Box {
    double lo[3], hi[3];
};

inline void Empty(Box& b)
{
    for (int k = 0; k < 3; ++k) { b.lo[k] = kInf; b.hi[k] = -kInf; }
}

inline void IncPt(Box& b, const double* p)
{
    for (int k = 0; k < 3; ++k) {
        if (p[k] < b.lo[k]) b.lo[k] = p[k];
        if (p[k] > b.hi[k]) b.hi[k] = p[k];
    }
}

inline void IncBox(Box& b, const Box& o)
{
    IncPt(b, o.lo);
    IncPt(b, o.hi);
}

inline double Area(const Box& b)
{
    const double ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
    if (ex < 0 || ey < 0 || ez < 0) return 0.0;
    return 2.0 * (ex * ey + ey * ez + ez * ex);
}

// Intermediate tree node built by workers before renumbering.
struct TNode {
    float bmin[3], bmax[3];
    uint32_t first;      // leaf: first prim slot
    uint32_t count;      // leaf prim count, 0 = internal
    uint8_t axis;
    int32_t left, right; // handles into the node pool (internal only)
};

struct Builder {
    const Box* primBox;
    const double* cen;  // 3 per prim
    uint32_t* idx;
    std::vector<TNode> pool;
    std::mutex poolMu;
    std::atomic<int> activeWorkers{0};
    int maxWorkers = 1;
    std::vector<std::thread> threads;
    std::mutex thrMu;

    int32_t Alloc()
    {
        std::lock_guard<std::mutex> g(poolMu);
        pool.emplace_back();
        return (int32_t)pool.size() - 1;
    }

    void SetBox(int32_t h, const Box& b)
    {
        std::lock_guard<std::mutex> g(poolMu);
        TNode& n = pool[h];
        for (int k = 0; k < 3; ++k) {
            n.bmin[k] = std::nextafter((float)b.lo[k], -FLT_MAX);
            n.bmax[k] = std::nextafter((float)b.hi[k], FLT_MAX);
        }
    }

    void SetLeaf(int32_t h, uint32_t first, uint32_t count)
    {
        std::lock_guard<std::mutex> g(poolMu);
        TNode& n = pool[h];
        n.first = first;
        n.count = count;
        n.axis = 0;
        n.left = n.right = -1;
    }

    void SetInner(int32_t h, uint8_t axis, int32_t l, int32_t r)
    {
        std::lock_guard<std::mutex> g(poolMu);
        TNode& n = pool[h];
        n.first = 0;
        n.count = 0;
        n.axis = axis;
        n.left = l;
        n.right = r;
    }

    void Recurse(int32_t h, uint32_t first, uint32_t last, const Box& cbox)
    {
        const uint32_t count = last - first;
        Box tight;
        Empty(tight);
        for (uint32_t i = first; i < last; ++i) IncBox(tight, primBox[idx[i]]);
        SetBox(h, tight);
        if (count <= 4) { SetLeaf(h, first, count); return; }

        const double ext[3] = {cbox.hi[0] - cbox.lo[0], cbox.hi[1] - cbox.lo[1], cbox.hi[2] - cbox.lo[2]};
        uint8_t axis = 0;
        if (ext[1] > ext[0]) axis = 1;
        if (ext[2] > ((axis == 0) ? ext[0] : ext[1])) axis = 2;
        const double cMin = cbox.lo[axis], cMax = cbox.hi[axis];
        if (cMax - cMin < 1e-12) { SetLeaf(h, first, count); return; }

        const int B = 32;
        Box bins[B];
        uint32_t bc[B];
        for (int i = 0; i < B; ++i) { Empty(bins[i]); bc[i] = 0; }
        const double invSpan = (double)B / (cMax - cMin);
        for (uint32_t i = first; i < last; ++i) {
            const double c = cen[3 * (size_t)idx[i] + axis];
            int bid = (int)((c - cMin) * invSpan);
            if (bid < 0) bid = 0;
            if (bid >= B) bid = B - 1;
            bc[bid]++;
            IncBox(bins[bid], primBox[idx[i]]);
        }
        Box lb[B - 1], rb[B - 1];
        uint32_t lc[B - 1], rc[B - 1];
        Box acc;
        Empty(acc);
        uint32_t n = 0;
        for (int i = 0; i + 1 < B; ++i) {
            if (bc[i] > 0) IncBox(acc, bins[i]);
            n += bc[i];
            lb[i] = acc;
            lc[i] = n;
        }
        Empty(acc);
        n = 0;
        for (int i = B - 1; i >= 1; --i) {
            if (bc[i] > 0) IncBox(acc, bins[i]);
            n += bc[i];
            rb[i - 1] = acc;
            rc[i - 1] = n;
        }
        const double parentArea = Area(tight);
        double bestCost = (double)count;
        int best = -1;
        for (int i = 0; i + 1 < B; ++i) {
            if (lc[i] == 0 || rc[i] == 0) continue;
            const double cost = 1.0 + 1.0 * ((Area(lb[i]) * (double)lc[i]) + (Area(rb[i]) * (double)rc[i])) / parentArea;
            if (cost < bestCost) { bestCost = cost; best = i; }
        }
        if (best < 0) { SetLeaf(h, first, count); return; }

        const double splitVal = cMin + (cMax - cMin) * (double)(best + 1) / (double)B;
        uint32_t mid = first;
        for (uint32_t i = first; i < last; ++i) {
            if (cen[3 * (size_t)idx[i] + axis] < splitVal) { std::swap(idx[i], idx[mid]); ++mid; }
        }
        if (mid == first || mid == last) {
            mid = first + count / 2;
            const double* c = cen;
            std::nth_element(idx + first, idx + mid, idx + last,
                             [c, axis](uint32_t a, uint32_t b) { return c[3 * (size_t)a + axis] < c[3 * (size_t)b + axis]; });
        }
        Box lcb, rcb;
        Empty(lcb);
        Empty(rcb);
        for (uint32_t i = first; i < mid; ++i) IncPt(lcb, &cen[3 * (size_t)idx[i]]);
        for (uint32_t i = mid; i < last; ++i) IncPt(rcb, &cen[3 * (size_t)idx[i]]);

        const int32_t l = Alloc(), r = Alloc();
        SetInner(h, axis, l, r);

        // Large right subtrees go to a worker thread; the partition ranges are
        // disjoint, so workers touch disjoint parts of idx.
        const uint32_t kParallelMin = 32768;
        if (last - mid >= kParallelMin && mid - first >= kParallelMin) {
            int cur = activeWorkers.load();
            while (cur < maxWorkers) {
                if (activeWorkers.compare_exchange_weak(cur, cur + 1)) {
                    {
                        std::lock_guard<std::mutex> g(thrMu);
                        threads.emplace_back([this, r, mid, last, rcb]() {
                            Recurse(r, mid, last, rcb);
                            activeWorkers.fetch_sub(1);
                        });
                    }
                    Recurse(l, first, mid, lcb);
                    return;
                }
            }
        }
        Recurse(l, first, mid, lcb);
        Recurse(r, mid, last, rcb);
    }
};

// Depth-first renumbering into the reference's allocation order.
void Renumber(const std::vector<TNode>& pool, int32_t h, uint32_t dst, std::vector<Node2>& out)
{
    // Iterative to avoid deep recursion on degenerate inputs.
    struct Item { int32_t h; uint32_t dst; };
    std::vector<Item> st;
    st.push_back({h, dst});
    // The reference allocates a node's child pair when the node is split,
    // then builds the whole left subtree (allocating its pairs) before the
    // right.  A pre-order walk that allocates each pair when its parent is
    // visited, visiting left before right, reproduces that order.
    while (!st.empty()) {
        Item it = st.back();
        st.pop_back();
        const TNode& n = pool[it.h];
        Node2& o = out[it.dst];
        for (int k = 0; k < 3; ++k) { o.bmin[k] = n.bmin[k]; o.bmax[k] = n.bmax[k]; }
        o.pad = 0;
        if (n.count > 0 || n.left < 0) {
            o.first_or_left = n.first;
            o.count = (uint16_t)n.count;
            o.axis = 0;
        } else {
            const uint32_t l = (uint32_t)out.size();
            out.emplace_back();
            out.emplace_back();
            Node2& o2 = out[it.dst];
            o2.first_or_left = l;
            o2.count = 0;
            o2.axis = n.axis;
            st.push_back({n.right, l + 1});
            st.push_back({n.left, l});
        }
    }
}

void InitEmpty4(Node4& n)
{
    for (int i = 0; i < 4; ++i) {
        n.minx[i] = n.miny[i] = n.minz[i] = FLT_MAX;
        n.maxx[i] = n.maxy[i] = n.maxz[i] = -FLT_MAX;
        n.child[i] = -1;
        n.count[i] = 0;
    }
    n.nchild = 0;
    n.axis = 0;
    std::memset(n.pad, 0, sizeof(n.pad));
}

void Slot(Node4& d, int i, const Node2& s)
{
    d.minx[i] = s.bmin[0]; d.miny[i] = s.bmin[1]; d.minz[i] = s.bmin[2];
    d.maxx[i] = s.bmax[0]; d.maxy[i] = s.bmax[1]; d.maxz[i] = s.bmax[2];
}

// BVH4 collapse in the reference's order (BVH.h:560-642): each internal
// BVH2 child contributes its two children; new BVH4 nodes are appended when
// first met, depth first.
void Collapse(const std::vector<Node2>& n2, std::vector<Node4>& n4)
{
    struct Item { uint32_t dst, src; };
    // Recursion order matters for numbering: the reference appends a child
    // node and immediately recurses into it before filling later slots.
    std::function<void(uint32_t, uint32_t)> rec = [&](uint32_t dst, uint32_t src) {
        const Node2 n = n2[src];
        const uint32_t l = n.first_or_left, r = l + 1;
        uint32_t cand[4];
        int nc = 0;
        if (n2[l].count > 0) cand[nc++] = l; else { cand[nc++] = n2[l].first_or_left; cand[nc++] = n2[l].first_or_left + 1; }
        if (n2[r].count > 0) cand[nc++] = r; else { cand[nc++] = n2[r].first_or_left; cand[nc++] = n2[r].first_or_left + 1; }
        n4[dst].nchild = (uint8_t)nc;
        n4[dst].axis = n.axis;
        for (int i = 0; i < nc; ++i) {
            const Node2 c = n2[cand[i]];
            if (c.count > 0) {
                Slot(n4[dst], i, c);
                n4[dst].child[i] = (int32_t)c.first_or_left;
                n4[dst].count[i] = c.count;
            } else {
                const uint32_t ci = (uint32_t)n4.size();
                n4.emplace_back();
                InitEmpty4(n4.back());
                rec(ci, cand[i]);
                Slot(n4[dst], i, c);
                n4[dst].child[i] = (int32_t)ci;
                n4[dst].count[i] = 0;
            }
        }
    };
    (void)sizeof(Item);
    n4.clear();
    if (n2.empty()) return;
    n4.reserve(n2.size() / 2 + 1);
    n4.emplace_back();
    InitEmpty4(n4[0]);
    if (n2[0].count > 0) {
        Slot(n4[0], 0, n2[0]);
        n4[0].child[0] = (int32_t)n2[0].first_or_left;
        n4[0].count[0] = n2[0].count;
        n4[0].nchild = 1;
        return;
    }
    rec(0, 0);
}

template <class F>
void ParallelFor(int64_t n, int threads, F fn)
{
    if (threads <= 1 || n < 65536) { fn(0, n); return; }
    std::vector<std::thread> ts;
    const int64_t chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int64_t s = t * chunk, e = std::min(n, s + chunk);
        if (s >= e) break;
        ts.emplace_back([=]() { fn(s, e); });
    }
    for (auto& t : ts) t.join();
}

}  // namespace

void BuildReferenceBVH(const float* tri9, int64_t n_tri, int threads, BuiltBVH& out)
{
    out.nodes2.clear();
    out.prims.clear();
    out.nodes4.clear();
    if (n_tri <= 0) return;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());

    std::vector<Box> primBox((size_t)n_tri);
    std::vector<double> cen(3 * (size_t)n_tri);
    ParallelFor(n_tri, threads, [&](int64_t s, int64_t e) {
        for (int64_t i = s; i < e; ++i) {
            Box b;
            Empty(b);
            for (int j = 0; j < 3; ++j) {
                const double p[3] = {tri9[9 * i + 3 * j], tri9[9 * i + 3 * j + 1], tri9[9 * i + 3 * j + 2]};
                IncPt(b, p);
            }
            primBox[i] = b;
            for (int k = 0; k < 3; ++k) cen[3 * i + k] = (b.lo[k] + b.hi[k]) * 0.5;
        }
    });
    Box rootC;
    Empty(rootC);
    for (int64_t i = 0; i < n_tri; ++i) IncPt(rootC, &cen[3 * i]);

    out.prims.resize((size_t)n_tri);
    for (int64_t i = 0; i < n_tri; ++i) out.prims[i] = (uint32_t)i;

    Builder b;
    b.primBox = primBox.data();
    b.cen = cen.data();
    b.idx = out.prims.data();
    b.maxWorkers = threads - 1;
    b.pool.reserve((size_t)n_tri);  // pool is mutex-guarded; reserve limits reallocation
    const int32_t root = b.Alloc();
    b.Recurse(root, 0, (uint32_t)n_tri, rootC);
    for (;;) {
        std::thread t;
        {
            std::lock_guard<std::mutex> g(b.thrMu);
            if (b.threads.empty()) break;
            t = std::move(b.threads.back());
            b.threads.pop_back();
        }
        t.join();
    }

    out.nodes2.reserve(b.pool.size());
    out.nodes2.emplace_back();
    Renumber(b.pool, root, 0, out.nodes2);
    Collapse(out.nodes2, out.nodes4);
}

bool ValidBVH2(const std::vector<Node2>& n2, size_t n_prims)
{
    if (n2.empty()) return false;
    std::vector<uint8_t> seen(n2.size(), 0);
    std::vector<std::pair<uint32_t, int>> stack = {{0u, 0}};
    seen[0] = 1;
    while (!stack.empty()) {
        const uint32_t i = stack.back().first;
        const int depth = stack.back().second;
        stack.pop_back();
        const Node2& n = n2[i];
        for (int k = 0; k < 3; ++k)
            if (!(n.bmin[k] <= n.bmax[k])) return false;   // inverted or NaN box
        if (n.count > 0) {
            if ((uint64_t)n.first_or_left + n.count > n_prims) return false;
            continue;
        }
        const uint64_t l = n.first_or_left;
        if (l <= i || l + 1 >= n2.size() || depth + 1 > kMaxBVH2Depth) return false;
        for (uint64_t c = l; c <= l + 1; ++c) {
            if (seen[c]) return false;
            seen[c] = 1;
            stack.push_back({(uint32_t)c, depth + 1});
        }
    }
    return true;
}

void MergeMeshBVHs(const std::vector<MeshBVH2>& meshes, BuiltBVH& out)
{
    out.nodes2.clear();
    out.prims.clear();
    out.nodes4.clear();
    if (meshes.empty()) return;
    std::vector<int64_t> base(meshes.size());   // leaf-order offset of each mesh
    for (size_t m = 0; m < meshes.size(); ++m) {
        base[m] = (int64_t)out.prims.size();
        for (uint32_t p : *meshes[m].prims) out.prims.push_back((uint32_t)(meshes[m].first + p));
    }
    // Copy mesh m's subtree rooted at `src` into slot `dst`, children pairs
    // appended depth first.
    std::function<void(size_t, uint32_t, uint32_t)> copy = [&](size_t m, uint32_t src, uint32_t dst) {
        Node2 n = (*meshes[m].nodes2)[src];
        if (n.count > 0) {
            n.first_or_left = (uint32_t)(n.first_or_left + base[m]);
            out.nodes2[dst] = n;
            return;
        }
        const uint32_t l = (uint32_t)out.nodes2.size();
        out.nodes2.resize(out.nodes2.size() + 2);
        const uint32_t sl = n.first_or_left;
        n.first_or_left = l;
        out.nodes2[dst] = n;
        copy(m, sl, l);
        copy(m, sl + 1, l + 1);
    };
    std::vector<uint32_t> order(meshes.size());
    for (size_t m = 0; m < meshes.size(); ++m) order[m] = (uint32_t)m;
    auto root_of = [&](uint32_t m) -> const Node2& { return (*meshes[m].nodes2)[0]; };
    // Top level over meshes order[lo, hi) into slot dst.
    std::function<void(size_t, size_t, uint32_t)> top = [&](size_t lo, size_t hi, uint32_t dst) {
        if (hi - lo == 1) {
            copy(order[lo], 0, dst);
            return;
        }
        Node2 n{};
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = 0; k < 3; ++k) { n.bmin[k] = INFINITY; n.bmax[k] = -INFINITY; }
        for (size_t i = lo; i < hi; ++i) {
            const Node2& r = root_of(order[i]);
            for (int k = 0; k < 3; ++k) {
                n.bmin[k] = std::min(n.bmin[k], r.bmin[k]);
                n.bmax[k] = std::max(n.bmax[k], r.bmax[k]);
                const float c = 0.5f * (r.bmin[k] + r.bmax[k]);
                clo[k] = std::min(clo[k], c);
                chi[k] = std::max(chi[k], c);
            }
        }
        int axis = 0;
        for (int k = 1; k < 3; ++k)
            if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
        const size_t mid = lo + (hi - lo) / 2;
        std::nth_element(order.begin() + lo, order.begin() + mid, order.begin() + hi, [&](uint32_t a, uint32_t b) {
            const float ca = root_of(a).bmin[axis] + root_of(a).bmax[axis];
            const float cb = root_of(b).bmin[axis] + root_of(b).bmax[axis];
            return ca < cb || (ca == cb && a < b);
        });
        const uint32_t l = (uint32_t)out.nodes2.size();
        out.nodes2.resize(out.nodes2.size() + 2);
        n.first_or_left = l;
        n.count = 0;
        n.axis = (uint8_t)axis;
        out.nodes2[dst] = n;
        top(lo, mid, l);
        top(mid, hi, l + 1);
    };
    size_t total = 1;
    for (const MeshBVH2& m : meshes) total += m.nodes2->size() + 1;
    out.nodes2.reserve(total);
    out.nodes2.emplace_back();
    top(0, meshes.size(), 0);
    Collapse(out.nodes2, out.nodes4);
}

std::vector<int32_t> BreadthFirstPositions(const BuiltBVH& b)
{
    const size_t n = b.nodes4.size();
    std::vector<int32_t> pos(n, -1);
    if (n == 0) return pos;
    std::vector<int32_t> q;
    q.reserve(n);
    q.push_back(0);
    for (size_t h = 0; h < q.size(); ++h) {
        const int32_t ni = q[h];
        pos[ni] = (int32_t)h;
        const Node4& s = b.nodes4[ni];
        for (int i = 0; i < s.nchild; ++i)
            if (s.count[i] == 0) q.push_back(s.child[i]);
    }
    return pos;
}

// Child link of slot i: the breadth-first position of an internal child, or
// ~first triangle of a leaf.
inline int32_t Link(const Node4& s, int i, const std::vector<int32_t>& pos)
{
    return s.count[i] > 0 ? ~s.child[i] : pos[s.child[i]];
}

void EncodeGpuNodes(const BuiltBVH& b, std::vector<GpuNode4>& out)
{
    out.resize(b.nodes4.size());
    const std::vector<int32_t> pos = BreadthFirstPositions(b);
    for (size_t n = 0; n < b.nodes4.size(); ++n) {
        const Node4& s = b.nodes4[n];
        GpuNode4& d = out[pos[n]];
        for (int i = 0; i < 4; ++i) {
            const bool valid = i < s.nchild;
            d.lox[i] = s.minx[i]; d.loy[i] = s.miny[i]; d.loz[i] = s.minz[i];
            d.hix[i] = s.maxx[i]; d.hiy[i] = s.maxy[i]; d.hiz[i] = s.maxz[i];
            d.child[i] = !valid ? INT32_MIN : Link(s, i, pos);
            d.count[i] = valid ? (int32_t)s.count[i] : -1;
        }
    }
}

namespace {

// Decode exactly as the traversal kernel does: origin + q * 2^e in FP32.
inline float Decode(float o, int e, int q)
{
    return o + (float)q * std::ldexp(1.0f, e);
}

}  // namespace

void EncodeQuantNodes(const BuiltBVH& b, std::vector<QNode4>& out)
{
    out.resize(b.nodes4.size());
    const std::vector<int32_t> pos = BreadthFirstPositions(b);
    for (size_t n = 0; n < b.nodes4.size(); ++n) {
        const Node4& s = b.nodes4[n];
        QNode4& d = out[pos[n]];
        std::memset(&d, 0, sizeof(d));
        d.nchild = s.nchild;
        const float* lo[3] = {s.minx, s.miny, s.minz};
        const float* hi[3] = {s.maxx, s.maxy, s.maxz};
        float org[3];
        int ex[3];
        for (int k = 0; k < 3; ++k) {
            float l = FLT_MAX, h = -FLT_MAX;
            for (int i = 0; i < s.nchild; ++i) { l = std::min(l, lo[k][i]); h = std::max(h, hi[k][i]); }
            org[k] = l;
            const double ext = (double)h - (double)l;
            // Smallest power of two with 254 * 2^e >= extent, leaving one
            // quantum of headroom for the outward nudge below.
            int e = -126;
            if (ext > 0) {
                e = (int)std::ceil(std::log2(ext / 254.0));
                while (254.0 * std::ldexp(1.0, e) < ext) ++e;
                if (e < -126) e = -126;
            }
            ex[k] = e;
        }
        d.ox = org[0]; d.oy = org[1]; d.oz = org[2];
        d.ex = (int8_t)ex[0]; d.ey = (int8_t)ex[1]; d.ez = (int8_t)ex[2];
        for (int i = 0; i < 4; ++i) {
            const bool valid = i < s.nchild;
            d.child[i] = !valid ? 0 : Link(s, i, pos);
            d.count[i] = valid ? (int16_t)std::min<int>(s.count[i], 32767) : (int16_t)-1;
            for (int k = 0; k < 3; ++k) {
                if (!valid) { d.qlo[k][i] = 255; d.qhi[k][i] = 0; continue; }
                const double sc = std::ldexp(1.0, ex[k]);
                int ql = (int)std::floor(((double)lo[k][i] - org[k]) / sc);
                int qh = (int)std::ceil(((double)hi[k][i] - org[k]) / sc);
                ql = std::max(0, std::min(255, ql));
                qh = std::max(0, std::min(255, qh));
                while (ql > 0 && Decode(org[k], ex[k], ql) >= lo[k][i]) --ql;
                while (qh < 255 && Decode(org[k], ex[k], qh) <= hi[k][i]) ++qh;
                d.qlo[k][i] = (uint8_t)ql;
                d.qhi[k][i] = (uint8_t)qh;
            }
        }
    }
}

float HalfToFloat(uint16_t h)
{
    const int sign = h >> 15, exp = (h >> 10) & 0x1f, man = h & 0x3ff;
    float v;
    if (exp == 0) v = std::ldexp((float)man, -24);                       // zero / subnormal
    else if (exp == 31) v = man ? std::numeric_limits<float>::quiet_NaN() : std::numeric_limits<float>::infinity();
    else v = std::ldexp((float)(man | 0x400), exp - 25);
    return sign ? -v : v;
}

uint16_t FloatToHalfDirected(float x, int dir)
{
    // Non-negative halves order like their bit patterns; find the largest
    // half <= |x| by binary search over 0x0000..0x7c00 (0 .. +inf).
    const float a = std::fabs(x);
    uint16_t lo = 0, hi = 0x7c00;
    while (lo < hi) {
        const uint16_t mid = (uint16_t)((lo + hi + 1) / 2);
        if (HalfToFloat(mid) <= a) lo = mid; else hi = (uint16_t)(mid - 1);
    }
    uint16_t mag = lo;   // largest half <= |x|
    const bool exact = HalfToFloat(mag) == a;
    // Rounding |x| down moves a positive x down and a negative x up.
    const bool wantDown = x >= 0.0f ? dir < 0 : dir > 0;
    if (!exact && !wantDown) mag = (uint16_t)(mag + 1);   // next half up (0x7c00 = inf at the top)
    return (uint16_t)((x < 0.0f ? 0x8000 : 0) | mag);
}

void EncodeHalfNodes(const BuiltBVH& b, std::vector<HNode4>& out)
{
    out.resize(b.nodes4.size());
    const std::vector<int32_t> pos = BreadthFirstPositions(b);
    for (size_t n = 0; n < b.nodes4.size(); ++n) {
        const Node4& s = b.nodes4[n];
        HNode4& d = out[pos[n]];
        for (int i = 0; i < 4; ++i) {
            const bool valid = i < s.nchild;
            // An empty slot gets the empty box (lo = +inf, hi = -inf).
            d.lox[i] = valid ? FloatToHalfDirected(s.minx[i], -1) : 0x7c00;
            d.loy[i] = valid ? FloatToHalfDirected(s.miny[i], -1) : 0x7c00;
            d.loz[i] = valid ? FloatToHalfDirected(s.minz[i], -1) : 0x7c00;
            d.hix[i] = valid ? FloatToHalfDirected(s.maxx[i], +1) : 0xfc00;
            d.hiy[i] = valid ? FloatToHalfDirected(s.maxy[i], +1) : 0xfc00;
            d.hiz[i] = valid ? FloatToHalfDirected(s.maxz[i], +1) : 0xfc00;
            d.child[i] = !valid ? INT32_MIN : Link(s, i, pos);
        }
    }
}

int TraceStackBound(const BuiltBVH& b)
{
    if (b.nodes4.empty()) return 0;
    int bound = 0;
    std::vector<std::pair<int32_t, int>> todo{{0, 0}};   // (node, entries deferred above it)
    while (!todo.empty()) {
        const auto [ni, above] = todo.back();
        todo.pop_back();
        const Node4& n = b.nodes4[ni];
        const int here = above + (n.nchild > 0 ? n.nchild - 1 : 0);
        bound = std::max(bound, here);
        for (int i = 0; i < n.nchild; ++i)
            if (n.count[i] == 0) todo.push_back({n.child[i], here});
    }
    return bound;
}

void EncodeTriangles(const float* tri9, const BuiltBVH& b, std::vector<GpuTri>& out)
{
    out.resize(b.prims.size());
    for (size_t i = 0; i < b.prims.size(); ++i) {
        const uint32_t p = b.prims[i];
        const float* s = tri9 + 9 * (size_t)p;
        GpuTri& t = out[i];
        for (int k = 0; k < 3; ++k) { t.v0[k] = s[k]; t.v1[k] = s[3 + k]; t.v2[k] = s[6 + k]; }
        std::memcpy(&t.v0[3], &p, 4);
        t.v1[3] = 0.0f;
        t.v2[3] = 0.0f;
    }
    // Mark the last triangle of every leaf (v1.w = 1) so the traversal can
    // walk a leaf from its first slot without a separate count.
    for (const Node4& n : b.nodes4)
        for (int i = 0; i < n.nchild; ++i)
            if (n.count[i] > 0) out[(size_t)n.child[i] + n.count[i] - 1].v1[3] = 1.0f;
}

}  // namespace rtb200
