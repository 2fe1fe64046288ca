// bvh_oracle.cpp -- TEST INFRASTRUCTURE ONLY (oracle port).
//
// A deliberately plain, single-threaded restatement of the reference
// renderer's BVH path, written for readability rather than speed:
//   * SAH-binned top-down BVH2 build   src/Library/Acceleration/BVH.h:772-1102
//   * BVH4 collapse                    BVH.h:477-642
//   * float slab test on 4 children    BVH.h:650-765 (scalar branch :738-763)
//   * float Moller-Trumbore filter     BVH.h:1111-1167
//   * closest-hit BVH4 traversal       BVH.h:1304-1370
//   * any-hit BVH4 traversal           BVH.h:1427-1471
//   * double Moller-Trumbore           src/Library/Intersection/RayTriangleIntersection.cpp:21-68
//   * leaf processor (both faces)      src/Library/Geometry/TriangleMeshGeometryIndexedSpecializations.h:116-183,478-525
// Compiled with -ffp-contract=off so float arithmetic rounds like the
// reference's SSE build.  Loaded only by tests, the smoke check and the CPU
// baseline leg of bench.py.

#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

const double kNearZero = 1e-12;            // Utilities/Math3D/Constants.h:33
const double kInf = DBL_MAX;               // RISE_INFINITY, Constants.h:34

struct Box { double lo[3], hi[3]; };

inline Box EmptyBox()
{
    Box b;
    for (int k = 0; k < 3; ++k) { b.lo[k] = kInf; b.hi[k] = -kInf; }
    return b;
}

// BoundingBox::Include(Point3) -- Utilities/BoundingBox.h:76-98
inline void IncludePoint(Box& b, const double p[3])
{
    for (int k = 0; k < 3; ++k) {
        if (p[k] < b.lo[k]) b.lo[k] = p[k];
        if (p[k] > b.hi[k]) b.hi[k] = p[k];
    }
}

inline void IncludeBox(Box& b, const Box& o)
{
    IncludePoint(b, o.lo);
    IncludePoint(b, o.hi);
}

// BVH.h:1083-1088
inline double SurfaceArea(const Box& b)
{
    const double ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
    if (ex < 0 || ey < 0 || ez < 0) return 0.0;
    return 2.0 * (ex * ey + ey * ez + ez * ex);
}

// BVH.h:1094-1102 -- outward rounding by one float ulp.
inline void SetNodeBox(orc_node2& n, const Box& b)
{
    for (int k = 0; k < 3; ++k) {
        n.bmin[k] = std::nextafter((float)b.lo[k], -FLT_MAX);
        n.bmax[k] = std::nextafter((float)b.hi[k], FLT_MAX);
    }
}

struct Bvh {
    std::vector<double> v;       // 9 doubles per triangle
    std::vector<orc_node2> nodes;
    std::vector<uint32_t> prims;
    std::vector<orc_node4> nodes4;
    std::vector<float> filt;     // 9 floats per reordered prim: p0, e1, e2
    // build scratch
    std::vector<Box> primBox;
    std::vector<double> cen;     // 3 per prim
};

void MakeLeaf(Bvh& b, uint32_t node, uint32_t first, uint32_t count)
{
    b.nodes[node].first_or_left = first;
    b.nodes[node].count = (uint16_t)count;
    b.nodes[node].axis = 0;
}

// BVH.h:860-1034
void BuildRecursive(Bvh& b, uint32_t node, std::vector<uint32_t>& idx, uint32_t first,
                    uint32_t last, const Box& cbox)
{
    const uint32_t count = last - first;
    Box tight = EmptyBox();
    for (uint32_t i = first; i < last; ++i) IncludeBox(tight, b.primBox[idx[i]]);
    SetNodeBox(b.nodes[node], tight);

    if (count <= 4) { MakeLeaf(b, node, first, count); return; }

    const double ext[3] = {cbox.hi[0] - cbox.lo[0], cbox.hi[1] - cbox.lo[1], cbox.hi[2] - cbox.lo[2]};
    uint8_t axis = 0;
    if (ext[1] > ext[0]) axis = 1;
    if (ext[2] > ((axis == 0) ? ext[0] : ext[1])) axis = 2;
    const double cMin = cbox.lo[axis], cMax = cbox.hi[axis];
    if (cMax - cMin < 1e-12) { MakeLeaf(b, node, first, count); return; }

    const uint32_t B = 32;
    Box binBox[32];
    uint32_t binCount[32];
    for (uint32_t i = 0; i < B; ++i) { binBox[i] = EmptyBox(); binCount[i] = 0; }
    const double invSpan = (double)B / (cMax - cMin);
    for (uint32_t i = first; i < last; ++i) {
        const double c = b.cen[3 * idx[i] + axis];
        int bid = (int)((c - cMin) * invSpan);
        if (bid < 0) bid = 0;
        if (bid >= (int)B) bid = B - 1;
        binCount[bid]++;
        IncludeBox(binBox[bid], b.primBox[idx[i]]);
    }

    Box leftBox[31], rightBox[31];
    uint32_t leftCount[31], rightCount[31];
    Box acc = EmptyBox();
    uint32_t accN = 0;
    for (uint32_t i = 0; i + 1 < B; ++i) {
        if (binCount[i] > 0) IncludeBox(acc, binBox[i]);
        accN += binCount[i];
        leftBox[i] = acc;
        leftCount[i] = accN;
    }
    acc = EmptyBox();
    accN = 0;
    for (int i = (int)B - 1; i >= 1; --i) {
        if (binCount[i] > 0) IncludeBox(acc, binBox[i]);
        accN += binCount[i];
        rightBox[i - 1] = acc;
        rightCount[i - 1] = accN;
    }

    const double parentArea = SurfaceArea(tight);
    const double leafCost = 1.0 * (double)count;
    double bestCost = leafCost;
    int bestSplit = -1;
    for (uint32_t i = 0; i + 1 < B; ++i) {
        if (leftCount[i] == 0 || rightCount[i] == 0) continue;
        const double cost = 1.0 + 1.0 * ((SurfaceArea(leftBox[i]) * (double)leftCount[i]) +
                                         (SurfaceArea(rightBox[i]) * (double)rightCount[i])) /
                                        parentArea;
        if (cost < bestCost) { bestCost = cost; bestSplit = (int)i; }
    }
    if (bestSplit < 0) { MakeLeaf(b, node, first, count); return; }

    const double splitVal = cMin + (cMax - cMin) * (double)(bestSplit + 1) / (double)B;
    uint32_t mid = first;
    for (uint32_t i = first; i < last; ++i) {
        if (b.cen[3 * idx[i] + axis] < splitVal) { std::swap(idx[i], idx[mid]); ++mid; }
    }
    if (mid == first || mid == last) {
        mid = first + count / 2;
        const std::vector<double>& cen = b.cen;
        std::nth_element(idx.begin() + first, idx.begin() + mid, idx.begin() + last,
                         [&](uint32_t x, uint32_t y) { return cen[3 * x + axis] < cen[3 * y + axis]; });
    }

    Box lc = EmptyBox(), rc = EmptyBox();
    for (uint32_t i = first; i < mid; ++i) IncludePoint(lc, &b.cen[3 * idx[i]]);
    for (uint32_t i = mid; i < last; ++i) IncludePoint(rc, &b.cen[3 * idx[i]]);

    const uint32_t left = (uint32_t)b.nodes.size();
    b.nodes.push_back(orc_node2{});
    b.nodes.push_back(orc_node2{});
    b.nodes[node].first_or_left = left;
    b.nodes[node].count = 0;
    b.nodes[node].axis = axis;
    BuildRecursive(b, left, idx, first, mid, lc);
    BuildRecursive(b, left + 1, idx, mid, last, rc);
}

void InitEmpty4(orc_node4& n)
{
    for (int i = 0; i < 4; ++i) {
        n.minx[i] = n.miny[i] = n.minz[i] = FLT_MAX;
        n.maxx[i] = n.maxy[i] = n.maxz[i] = -FLT_MAX;
        n.child[i] = -1;
        n.count[i] = 0;
    }
    n.nchild = 0;
    n.axis = 0;
    for (int i = 0; i < 6; ++i) n.pad[i] = 0;
}

void SetSlot(Bvh& b, uint32_t dst, int i, const orc_node2& s)
{
    orc_node4& d = b.nodes4[dst];
    d.minx[i] = s.bmin[0]; d.miny[i] = s.bmin[1]; d.minz[i] = s.bmin[2];
    d.maxx[i] = s.bmax[0]; d.maxy[i] = s.bmax[1]; d.maxz[i] = s.bmax[2];
}

// BVH.h:560-642
void Collapse(Bvh& b, uint32_t dst, uint32_t src)
{
    const orc_node2 n = b.nodes[src];
    const uint32_t l = n.first_or_left, r = l + 1;
    uint32_t cand[4];
    int nc = 0;
    if (b.nodes[l].count > 0) cand[nc++] = l;
    else { cand[nc++] = b.nodes[l].first_or_left; cand[nc++] = b.nodes[l].first_or_left + 1; }
    if (b.nodes[r].count > 0) cand[nc++] = r;
    else { cand[nc++] = b.nodes[r].first_or_left; cand[nc++] = b.nodes[r].first_or_left + 1; }
    b.nodes4[dst].nchild = (uint8_t)nc;
    b.nodes4[dst].axis = n.axis;
    for (int i = 0; i < nc; ++i) {
        const orc_node2 c = b.nodes[cand[i]];
        if (c.count > 0) {
            SetSlot(b, dst, i, c);
            b.nodes4[dst].child[i] = (int32_t)c.first_or_left;
            b.nodes4[dst].count[i] = c.count;
        } else {
            const uint32_t ci = (uint32_t)b.nodes4.size();
            b.nodes4.push_back(orc_node4{});
            InitEmpty4(b.nodes4.back());
            Collapse(b, ci, cand[i]);
            SetSlot(b, dst, i, c);
            b.nodes4[dst].child[i] = (int32_t)ci;
            b.nodes4[dst].count[i] = 0;
        }
    }
}

// BVH.h:477-519
void BuildBVH4(Bvh& b)
{
    b.nodes4.clear();
    if (b.nodes.empty()) return;
    b.nodes4.push_back(orc_node4{});
    InitEmpty4(b.nodes4[0]);
    const orc_node2 root = b.nodes[0];
    if (root.count > 0) {
        SetSlot(b, 0, 0, root);
        b.nodes4[0].child[0] = (int32_t)root.first_or_left;
        b.nodes4[0].count[0] = root.count;
        b.nodes4[0].nchild = 1;
        return;
    }
    Collapse(b, 0, 0);
}

// RayTriangleIntersection.cpp:21-68 (double precision, NEARZERO slack).
int RayTri(const double o[3], const double d[3], const double v0[3], const double ea[3],
           const double eb[3], double* t, double* alpha, double* beta)
{
    const double pv[3] = {d[1] * eb[2] - d[2] * eb[1], d[2] * eb[0] - d[0] * eb[2], d[0] * eb[1] - d[1] * eb[0]};
    const double det = ea[0] * pv[0] + ea[1] * pv[1] + ea[2] * pv[2];
    *t = kInf;
    if (det > -kNearZero && det < kNearZero) return 0;
    const double oodet = 1.0 / det;
    const double tv[3] = {o[0] - v0[0], o[1] - v0[1], o[2] - v0[2]};
    const double a = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * oodet;
    if ((a < 0.0 - kNearZero) || (a > 1.0 + kNearZero)) return 0;
    const double qv[3] = {tv[1] * ea[2] - tv[2] * ea[1], tv[2] * ea[0] - tv[0] * ea[2], tv[0] * ea[1] - tv[1] * ea[0]};
    const double bb = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * oodet;
    if ((bb < 0.0 - kNearZero) || ((a + bb) > 1.0 + kNearZero)) return 0;
    const double tt = (eb[0] * qv[0] + eb[1] * qv[1] + eb[2] * qv[2]) * oodet;
    *t = tt;
    if (tt >= kNearZero) { *alpha = a; *beta = bb; return 1; }
    return 0;
}

// BVH.h:1111-1167
bool FloatFilter(const float o[3], const float d[3], const float* f, float best, float* tOut)
{
    const float EPS = 1e-5f;
    const float* p0 = f; const float* e1 = f + 3; const float* e2 = f + 6;
    const float pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
    const float det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
    if (std::fabs(det) < 1e-20f) return false;
    const float invDet = 1.0f / det;
    const float tv[3] = {o[0] - p0[0], o[1] - p0[1], o[2] - p0[2]};
    const float u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * invDet;
    if (u < -EPS || u > 1.0f + EPS) return false;
    const float qv[3] = {tv[1] * e1[2] - tv[2] * e1[1], tv[2] * e1[0] - tv[0] * e1[2], tv[0] * e1[1] - tv[1] * e1[0]};
    const float v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * invDet;
    if (v < -EPS || u + v > 1.0f + EPS) return false;
    const float t = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * invDet;
    if (t < -EPS || t > best + EPS) return false;
    *tOut = t;
    return true;
}

// BVH.h:738-763 (scalar branch of RayBox4; the SSE/NEON branches compute the
// same IEEE single-precision values).
uint32_t RayBox4(const float o[3], const float inv[3], float best, const orc_node4& n, float te[4])
{
    uint32_t mask = 0;
    for (int i = 0; i < 4; ++i) {
        const float t1x = (n.minx[i] - o[0]) * inv[0], t2x = (n.maxx[i] - o[0]) * inv[0];
        const float t1y = (n.miny[i] - o[1]) * inv[1], t2y = (n.maxy[i] - o[1]) * inv[1];
        const float t1z = (n.minz[i] - o[2]) * inv[2], t2z = (n.maxz[i] - o[2]) * inv[2];
        float tmin = std::fmax(std::fmax(std::fmin(t1x, t2x), std::fmin(t1y, t2y)), std::fmin(t1z, t2z));
        float tmax = std::fmin(std::fmin(std::fmax(t1x, t2x), std::fmax(t1y, t2y)), std::fmax(t1z, t2z));
        tmin = std::fmax(tmin, 0.0f);
        tmax = std::fmin(tmax, best);
        if (tmin <= tmax) { te[i] = tmin; mask |= 1u << i; }
        else te[i] = FLT_MAX;
    }
    return mask;
}

// BVH.h:1212-1225
void PrepRay(const float* r, float o[3], float d[3], float inv[3])
{
    for (int k = 0; k < 3; ++k) {
        o[k] = r[k];
        d[k] = r[4 + k];
        inv[k] = (d[k] == 0.0f) ? ((d[k] >= 0) ? FLT_MAX : -FLT_MAX) : 1.0f / d[k];
    }
}

inline void TriEdges(const Bvh& b, uint32_t tri, double v0[3], double ea[3], double eb[3])
{
    const double* p = &b.v[9ull * tri];
    for (int k = 0; k < 3; ++k) { v0[k] = p[k]; ea[k] = p[3 + k] - p[k]; eb[k] = p[6 + k] - p[k]; }
}

double PointSegDist(const double p[3], const double a[3], const double c[3])
{
    double ab[3], ap[3];
    for (int k = 0; k < 3; ++k) { ab[k] = c[k] - a[k]; ap[k] = p[k] - a[k]; }
    const double l2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    double s = l2 > 0 ? (ap[0] * ab[0] + ap[1] * ab[1] + ap[2] * ab[2]) / l2 : 0.0;
    s = s < 0 ? 0 : (s > 1 ? 1 : s);
    double dd = 0;
    for (int k = 0; k < 3; ++k) { const double e = a[k] + s * ab[k] - p[k]; dd += e * e; }
    return std::sqrt(dd);
}

// Distance from the hit point to the nearest edge of the hit triangle.
double EdgeDistance(const double* tri, const double o[3], const double d[3], double t)
{
    const double p[3] = {o[0] + t * d[0], o[1] + t * d[1], o[2] + t * d[2]};
    const double d0 = PointSegDist(p, tri, tri + 3);
    const double d1 = PointSegDist(p, tri + 3, tri + 6);
    const double d2 = PointSegDist(p, tri + 6, tri);
    return std::min(d0, std::min(d1, d2));
}

// Closest hit -- BVH.h:1304-1370 with leaf processing BVH.h:1237-1255.
void Closest(const Bvh& b, const float* r, int32_t* idOut, double* tOut, double* eOut)
{
    *idOut = -1; *tOut = -1.0; if (eOut) *eOut = -1.0;
    if (b.nodes4.empty()) return;
    float o[3], d[3], inv[3];
    PrepRay(r, o, d, inv);
    const double od[3] = {r[0], r[1], r[2]}, dd[3] = {r[4], r[5], r[6]};
    double range = kInf;
    int32_t best = -1;
    std::vector<uint32_t> stack;
    stack.push_back(0);
    while (!stack.empty()) {
        const uint32_t ni = stack.back();
        stack.pop_back();
        const orc_node4& n = b.nodes4[ni];
        float te[4];
        const uint32_t mask = RayBox4(o, inv, (float)range, n, te) & ((1u << n.nchild) - 1u);
        if (!mask) continue;
        int order[4], nh = 0;
        for (int i = 0; i < 4; ++i) if (mask & (1u << i)) order[nh++] = i;
        for (int a = 0; a < nh - 1; ++a) {
            int mx = a;
            for (int c = a + 1; c < nh; ++c) if (te[order[c]] > te[order[mx]]) mx = c;
            if (mx != a) std::swap(order[a], order[mx]);
        }
        for (int h = 0; h < nh; ++h) {
            const int i = order[h];
            if (n.count[i] > 0) {
                const uint32_t s = (uint32_t)n.child[i], e = s + n.count[i];
                for (uint32_t p = s; p < e; ++p) {
                    float ft;
                    if (!FloatFilter(o, d, &b.filt[9ull * p], (float)range, &ft)) continue;
                    double v0[3], ea[3], eb[3], t, al, be;
                    TriEdges(b, b.prims[p], v0, ea, eb);
                    if (RayTri(od, dd, v0, ea, eb, &t, &al, &be) && t < range) {
                        range = t;
                        best = (int32_t)b.prims[p];
                    }
                }
            } else {
                stack.push_back((uint32_t)n.child[i]);
            }
        }
    }
    if (best >= 0) {
        *idOut = best;
        *tOut = range;
        if (eOut) *eOut = EdgeDistance(&b.v[9ull * best], od, dd, range);
    }
}

// Any hit -- BVH.h:1427-1471 with the leaf test at BVH.h:1278-1301 and the
// processor's (0, dHowFar) acceptance, Specializations.h:515-520.
bool Any(const Bvh& b, const float* r)
{
    if (b.nodes4.empty()) return false;
    float o[3], d[3], inv[3];
    PrepRay(r, o, d, inv);
    const double od[3] = {r[0], r[1], r[2]}, dd[3] = {r[4], r[5], r[6]};
    const double howFar = (double)r[7];
    const float best = (float)howFar;
    std::vector<uint32_t> stack;
    stack.push_back(0);
    while (!stack.empty()) {
        const uint32_t ni = stack.back();
        stack.pop_back();
        const orc_node4& n = b.nodes4[ni];
        float te[4];
        const uint32_t mask = RayBox4(o, inv, best, n, te) & ((1u << n.nchild) - 1u);
        if (!mask) continue;
        for (int i = 0; i < 4; ++i) {
            if (!(mask & (1u << i))) continue;
            if (n.count[i] > 0) {
                const uint32_t s = (uint32_t)n.child[i], e = s + n.count[i];
                for (uint32_t p = s; p < e; ++p) {
                    float ft;
                    if (!FloatFilter(o, d, &b.filt[9ull * p], best, &ft)) continue;
                    double v0[3], ea[3], eb[3], t, al, be;
                    TriEdges(b, b.prims[p], v0, ea, eb);
                    if (RayTri(od, dd, v0, ea, eb, &t, &al, &be) && t > kNearZero && t < howFar) return true;
                }
            } else {
                stack.push_back((uint32_t)n.child[i]);
            }
        }
    }
    return false;
}

// Double-precision ray variants for the path-tracing oracle: the reference
// casts double rays; the traversal rounds them to float for the node tests
// (BVH.h:1212-1225) and certifies leaves in double.
int32_t ClosestD(const Bvh& b, const double od[3], const double dd[3], double* tOut)
{
    const float r[8] = {(float)od[0], (float)od[1], (float)od[2], 0.0f, (float)dd[0], (float)dd[1], (float)dd[2], 0.0f};
    float o[3], d[3], inv[3];
    PrepRay(r, o, d, inv);
    double range = kInf;
    int32_t best = -1;
    if (b.nodes4.empty()) return -1;
    std::vector<uint32_t> stack;
    stack.push_back(0);
    while (!stack.empty()) {
        const uint32_t ni = stack.back();
        stack.pop_back();
        const orc_node4& n = b.nodes4[ni];
        float te[4];
        const uint32_t mask = RayBox4(o, inv, (float)range, n, te) & ((1u << n.nchild) - 1u);
        if (!mask) continue;
        for (int i = 0; i < 4; ++i) {
            if (!(mask & (1u << i))) continue;
            if (n.count[i] > 0) {
                const uint32_t s = (uint32_t)n.child[i], e = s + n.count[i];
                for (uint32_t p = s; p < e; ++p) {
                    float ft;
                    if (!FloatFilter(o, d, &b.filt[9ull * p], (float)range, &ft)) continue;
                    double v0[3], ea[3], eb[3], t, al, be;
                    TriEdges(b, b.prims[p], v0, ea, eb);
                    if (RayTri(od, dd, v0, ea, eb, &t, &al, &be) && t < range) { range = t; best = (int32_t)b.prims[p]; }
                }
            } else {
                stack.push_back((uint32_t)n.child[i]);
            }
        }
    }
    *tOut = range;
    return best;
}

bool AnyD(const Bvh& b, const double od[3], const double dd[3], double howFar)
{
    float r[8] = {(float)od[0], (float)od[1], (float)od[2], 0.0f, (float)dd[0], (float)dd[1], (float)dd[2], (float)howFar};
    float o[3], d[3], inv[3];
    PrepRay(r, o, d, inv);
    const float best = (float)howFar;
    if (b.nodes4.empty()) return false;
    std::vector<uint32_t> stack;
    stack.push_back(0);
    while (!stack.empty()) {
        const uint32_t ni = stack.back();
        stack.pop_back();
        const orc_node4& n = b.nodes4[ni];
        float te[4];
        const uint32_t mask = RayBox4(o, inv, best, n, te) & ((1u << n.nchild) - 1u);
        if (!mask) continue;
        for (int i = 0; i < 4; ++i) {
            if (!(mask & (1u << i))) continue;
            if (n.count[i] > 0) {
                const uint32_t s = (uint32_t)n.child[i], e = s + n.count[i];
                for (uint32_t p = s; p < e; ++p) {
                    float ft;
                    if (!FloatFilter(o, d, &b.filt[9ull * p], best, &ft)) continue;
                    double v0[3], ea[3], eb[3], t, al, be;
                    TriEdges(b, b.prims[p], v0, ea, eb);
                    if (RayTri(od, dd, v0, ea, eb, &t, &al, &be) && t > kNearZero && t < howFar) return true;
                }
            } else {
                stack.push_back((uint32_t)n.child[i]);
            }
        }
    }
    return false;
}

template <class F>
void Parallel(int64_t n, int threads, F fn)
{
    if (threads <= 1 || n < 2048) { fn(0, n); return; }
    std::atomic<int64_t> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                const int64_t s = next.fetch_add(2048);
                if (s >= n) break;
                fn(s, std::min<int64_t>(n, s + 2048));
            }
        });
    for (auto& th : pool) th.join();
}

}  // namespace

struct orc_bvh { Bvh b; };

int32_t orc_closest_d(const orc_bvh* h, const double o[3], const double d[3], double* t)
{
    return ClosestD(h->b, o, d, t);
}

bool orc_any_d(const orc_bvh* h, const double o[3], const double d[3], double tmax)
{
    return AnyD(h->b, o, d, tmax);
}

extern "C" {

// BVH.h:162-192 (constructor: Build, BuildFastFilter, BuildBVH4) with the
// triangle-mesh configuration leaf 4, 32 bins, Ctrav = Cint = 1
// (src/Library/Geometry/TriangleMeshGeometryIndexed.cpp:529-535).
orc_bvh* orc_bvh_build(const float* tri9, int64_t n_tri)
{
    orc_bvh* h = new orc_bvh();
    Bvh& b = h->b;
    b.v.assign(tri9, tri9 + 9 * n_tri);
    if (n_tri == 0) return h;
    b.primBox.resize((size_t)n_tri);
    b.cen.resize(3 * (size_t)n_tri);
    Box rootC = EmptyBox();
    for (int64_t i = 0; i < n_tri; ++i) {
        Box bb = EmptyBox();
        for (int j = 0; j < 3; ++j) IncludePoint(bb, &b.v[9 * i + 3 * j]);
        b.primBox[i] = bb;
        for (int k = 0; k < 3; ++k) b.cen[3 * i + k] = (bb.lo[k] + bb.hi[k]) * 0.5;
        IncludePoint(rootC, &b.cen[3 * i]);
    }
    b.nodes.reserve(2 * (size_t)n_tri);
    b.nodes.push_back(orc_node2{});
    std::vector<uint32_t> idx((size_t)n_tri);
    for (int64_t i = 0; i < n_tri; ++i) idx[i] = (uint32_t)i;
    BuildRecursive(b, 0, idx, 0, (uint32_t)n_tri, rootC);
    b.prims = idx;
    // BVH.h:431-467 -- float (p0, e1, e2) per reordered prim.
    b.filt.resize(9 * (size_t)n_tri);
    for (int64_t i = 0; i < n_tri; ++i) {
        float v[9];
        for (int k = 0; k < 9; ++k) v[k] = (float)b.v[9ull * b.prims[i] + k];
        for (int k = 0; k < 3; ++k) {
            b.filt[9 * i + k] = v[k];
            b.filt[9 * i + 3 + k] = v[3 + k] - v[k];
            b.filt[9 * i + 6 + k] = v[6 + k] - v[k];
        }
    }
    BuildBVH4(b);
    b.primBox.clear(); b.primBox.shrink_to_fit();
    b.cen.clear(); b.cen.shrink_to_fit();
    return h;
}

void orc_bvh_destroy(orc_bvh* b) { delete b; }
int64_t orc_bvh_num_nodes2(const orc_bvh* b) { return (int64_t)b->b.nodes.size(); }
int64_t orc_bvh_num_nodes4(const orc_bvh* b) { return (int64_t)b->b.nodes4.size(); }

void orc_bvh_export(const orc_bvh* h, orc_node2* nodes2, uint32_t* prims, orc_node4* nodes4)
{
    const Bvh& b = h->b;
    if (nodes2 && !b.nodes.empty()) std::memcpy(nodes2, b.nodes.data(), b.nodes.size() * sizeof(orc_node2));
    if (prims && !b.prims.empty()) std::memcpy(prims, b.prims.data(), b.prims.size() * 4);
    if (nodes4 && !b.nodes4.empty()) std::memcpy(nodes4, b.nodes4.data(), b.nodes4.size() * sizeof(orc_node4));
}

void orc_closest(const orc_bvh* h, const float* rays, int64_t n, int32_t* id, double* t,
                 double* edge, int threads)
{
    Parallel(n, threads, [&](int64_t s, int64_t e) {
        for (int64_t i = s; i < e; ++i) Closest(h->b, rays + 8 * i, id + i, t + i, edge ? edge + i : nullptr);
    });
}

void orc_any(const orc_bvh* h, const float* rays, int64_t n, uint8_t* occ, int threads)
{
    Parallel(n, threads, [&](int64_t s, int64_t e) {
        for (int64_t i = s; i < e; ++i) occ[i] = Any(h->b, rays + 8 * i) ? 1 : 0;
    });
}

void orc_closest_brute(const float* tri9, int64_t n_tri, const float* rays, int64_t n,
                       int32_t* id, double* t)
{
    for (int64_t i = 0; i < n; ++i) {
        const float* r = rays + 8 * i;
        const double o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
        double best = kInf;
        int32_t bi = -1;
        for (int64_t k = 0; k < n_tri; ++k) {
            const float* p = tri9 + 9 * k;
            const double v0[3] = {p[0], p[1], p[2]};
            const double ea[3] = {(double)p[3] - p[0], (double)p[4] - p[1], (double)p[5] - p[2]};
            const double eb[3] = {(double)p[6] - p[0], (double)p[7] - p[1], (double)p[8] - p[2]};
            double tt, al, be;
            if (RayTri(o, d, v0, ea, eb, &tt, &al, &be) && tt < best) { best = tt; bi = (int32_t)k; }
        }
        id[i] = bi;
        t[i] = bi >= 0 ? best : -1.0;
    }
}

int orc_ray_triangle(const double* o, const double* d, const double* v0, const double* ea,
                     const double* eb, double* t, double* alpha, double* beta)
{
    *alpha = 0; *beta = 0;
    return RayTri(o, d, v0, ea, eb, t, alpha, beta);
}

}  // extern "C"
