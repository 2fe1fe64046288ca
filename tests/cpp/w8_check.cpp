// w8_check.cpp -- host check of the eight-wide node encoding (bvh_wide.cpp).
//
// Builds the reference BVH over a triangle file, encodes the eight-wide
// layout and checks, on the host:
//  * every input triangle appears exactly once in the layout's triangle order;
//  * links and triangle runs stay inside their arrays, internal children
//    follow their parent (breadth-first), meta offsets fit the 24-bit mask;
//  * every decoded 8-bit child box contains, in FP32, every triangle below it;
//  * a traversal with the device's group and octant rules (in double
//    precision) finds, for every ray, the closest triangle a brute-force
//    test over all triangles finds (or an equally distant one).
// Usage: w8_check tri.bin rays.bin  (float32 arrays: n x 9 and m x 8).
// Prints "ok <nodes> <depth>" or the first failure; exit status 0 on success.
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <vector>

#include "bvh_build.h"

using namespace rtb200;

static std::vector<float> ReadAll(const char* path)
{
    std::vector<float> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)n / 4);
    if (std::fread(v.data(), 4, v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

static float Dec(float o, int e, int q) { return o + (float)q * std::ldexp(1.0f, e); }

struct Box { float lo[3], hi[3]; };

static bool Fail(const char* what, long a = 0, long b = 0)
{
    std::printf("FAIL %s %ld %ld\n", what, a, b);
    return false;
}

// Double-precision Moller-Trumbore (the reference's test) for the checker.
static bool Hit(const float* t9, const double* o, const double* d, double& t)
{
    const double a[3] = {t9[0], t9[1], t9[2]};
    const double e1[3] = {t9[3] - a[0], t9[4] - a[1], t9[5] - a[2]};
    const double e2[3] = {t9[6] - a[0], t9[7] - a[1], t9[8] - a[2]};
    const double pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
    const double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
    if (std::fabs(det) < 1e-12) return false;
    const double inv = 1.0 / det;
    const double tv[3] = {o[0] - a[0], o[1] - a[1], o[2] - a[2]};
    const double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * inv;
    if (u < -1e-12 || u > 1.0 + 1e-12) return false;
    const double qv[3] = {tv[1] * e1[2] - tv[2] * e1[1], tv[2] * e1[0] - tv[0] * e1[2], tv[0] * e1[1] - tv[1] * e1[0]};
    const double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv;
    if (v < -1e-12 || u + v > 1.0 + 1e-12) return false;
    t = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv;
    return t > 1e-12;
}

int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    const std::vector<float> tri9 = ReadAll(argv[1]);
    const std::vector<float> rays = ReadAll(argv[2]);
    const int64_t n_tri = (int64_t)(tri9.size() / 9);
    BuiltBVH b;
    BuildReferenceBVH(tri9.data(), n_tri, 0, b);
    std::vector<WNode8> nodes;
    std::vector<uint32_t> prims;
    int depth = 0;
    if (!EncodeWideNodes(b, nodes, prims, depth)) return Fail("encode") ? 0 : 1;
    // Each triangle once.
    std::vector<int> seen(n_tri, 0);
    for (uint32_t p : prims) {
        if (p >= (uint32_t)n_tri) return Fail("prim range", p) ? 0 : 1;
        ++seen[p];
    }
    for (int64_t i = 0; i < n_tri; ++i)
        if (seen[i] != 1) return Fail("prim count", i, seen[i]) ? 0 : 1;
    // Structure and conservative boxes (bottom-up triangle bounds per node).
    std::vector<Box> sub(nodes.size());
    for (int64_t ni = (int64_t)nodes.size() - 1; ni >= 0; --ni) {
        const WNode8& n = nodes[ni];
        Box u{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
        const float org[3] = {n.px, n.py, n.pz};
        const int ex[3] = {n.ex, n.ey, n.ez};
        const uint8_t* ql[3] = {n.qlox, n.qloy, n.qloz};
        const uint8_t* qh[3] = {n.qhix, n.qhiy, n.qhiz};
        int rank = 0;
        for (int s = 0; s < 8; ++s) {
            Box c{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
            bool any = false;
            if ((n.imask >> s) & 1) {
                const uint32_t ci = n.child_base + rank++;
                if (ci <= (uint32_t)ni || ci >= nodes.size()) return Fail("child link", ni, ci) ? 0 : 1;
                c = sub[ci];
                any = true;
            } else if (n.meta[s]) {
                const unsigned off = n.meta[s] & 31u, bits = n.meta[s] >> 5;
                if (bits != 1 && bits != 3 && bits != 7) return Fail("meta count", ni, s) ? 0 : 1;
                const unsigned cnt = bits == 1 ? 1 : (bits == 3 ? 2 : 3);
                if (off + cnt > 24 || n.tri_base + off + cnt > prims.size()) return Fail("meta range", ni, s) ? 0 : 1;
                for (unsigned t = 0; t < cnt; ++t) {
                    const float* v = &tri9[9 * (size_t)prims[n.tri_base + off + t]];
                    for (int j = 0; j < 9; ++j) {
                        c.lo[j % 3] = std::fmin(c.lo[j % 3], v[j]);
                        c.hi[j % 3] = std::fmax(c.hi[j % 3], v[j]);
                    }
                }
                any = true;
            }
            if (!any) continue;
            for (int k = 0; k < 3; ++k) {
                if (!(Dec(org[k], ex[k], ql[k][s]) <= c.lo[k]) || !(Dec(org[k], ex[k], qh[k][s]) >= c.hi[k]))
                    return Fail("box not conservative", ni, s) ? 0 : 1;
                u.lo[k] = std::fmin(u.lo[k], c.lo[k]);
                u.hi[k] = std::fmax(u.hi[k], c.hi[k]);
            }
        }
        sub[ni] = u;
    }
    // Traversal with the device's rules against brute force.
    const size_t n_rays = rays.size() / 8;
    for (size_t r = 0; r < n_rays; ++r) {
        const float* R = &rays[8 * r];
        const double o[3] = {R[0], R[1], R[2]}, d[3] = {R[4], R[5], R[6]};
        double bt = R[7];
        long best = -1;
        for (int64_t i = 0; i < n_tri; ++i) {
            double t;
            if (Hit(&tri9[9 * i], o, d, t) && t > R[3] && t < bt) { bt = t; best = (long)i; }
        }
        const unsigned oct = (d[0] >= 0 ? 1u : 0u) | (d[1] >= 0 ? 2u : 0u) | (d[2] >= 0 ? 4u : 0u);
        std::vector<std::pair<uint32_t, uint32_t>> stack;
        std::pair<uint32_t, uint32_t> ng{0u, (1u << (24 + oct)) | 1u};
        double gt = R[7];
        long gbest = -1;
        for (int guard = 0; guard < 10000000; ++guard) {
            uint32_t tbase = 0, tmask = 0;
            if (ng.second & 0xff000000u) {
                const unsigned j = (unsigned)__builtin_ctz(ng.second >> 24);
                ng.second &= ~(1u << (24 + j));
                const unsigned slot = j ^ oct;
                const uint32_t ni = ng.first + (uint32_t)__builtin_popcount(ng.second & 0xffu & ((1u << slot) - 1u));
                if (ng.second & 0xff000000u) stack.push_back(ng);
                const WNode8& n = nodes[ni];
                const float org[3] = {n.px, n.py, n.pz};
                const int ex[3] = {n.ex, n.ey, n.ez};
                const uint8_t* ql[3] = {n.qlox, n.qloy, n.qloz};
                const uint8_t* qh[3] = {n.qhix, n.qhiy, n.qhiz};
                uint32_t hn = 0, ht = 0;
                for (int s = 0; s < 8; ++s) {
                    double tn = R[3], tf = gt;
                    for (int k = 0; k < 3; ++k) {
                        const double lo = Dec(org[k], ex[k], ql[k][s]), hi = Dec(org[k], ex[k], qh[k][s]);
                        if (d[k] == 0.0) {
                            if (o[k] < lo || o[k] > hi) tf = -1.0;
                            continue;
                        }
                        double a = (lo - o[k]) / d[k], c = (hi - o[k]) / d[k];
                        if (a > c) std::swap(a, c);
                        tn = std::fmax(tn, a);
                        tf = std::fmin(tf, c);
                    }
                    if (!(tn <= tf * (1 + 1e-9) + 1e-12)) continue;
                    if ((n.imask >> s) & 1) hn |= 1u << (24 + (s ^ oct));
                    else ht |= (uint32_t)(n.meta[s] >> 5) << (n.meta[s] & 31u);
                }
                ng = {n.child_base, hn | n.imask};
                tbase = n.tri_base;
                tmask = ht;
            }
            while (tmask) {
                const unsigned k = (unsigned)__builtin_ctz(tmask);
                tmask &= tmask - 1;
                const uint32_t p = prims[tbase + k];
                double t;
                if (Hit(&tri9[9 * (size_t)p], o, d, t) && t > R[3] && t < gt) { gt = t; gbest = (long)p; }
            }
            if (!(ng.second & 0xff000000u)) {
                if (stack.empty()) break;
                ng = stack.back();
                stack.pop_back();
            }
            if ((long)stack.size() > depth) return Fail("stack deeper than the levels", (long)r, (long)stack.size()) ? 0 : 1;
        }
        if (gbest != best && !(best >= 0 && gbest >= 0 && gt == bt)) return Fail("closest hit", (long)r, gbest) ? 0 : 1;
    }
    // The device loop as a warp executes it (TraceW8, raycast.cuh): 32 lanes in
    // lockstep, a lane postponing its triangle group while fewer than 8 lanes
    // of the warp test triangles, it still has a node group to continue with
    // and the stack keeps room for one node group per level; every ray must
    // finish within a step bound and find the same closest hit.
    const int kStack = 24, kLevels = 12, kTriLanes = 8;
    struct Lane {
        double o[3], d[3], tmin, best;
        unsigned oct;
        std::pair<uint32_t, uint32_t> ng, tg;
        std::vector<std::pair<uint32_t, uint32_t>> stk;
        long bestp;
        bool done;
        size_t ray;
    };
    for (size_t r0 = 0; r0 < n_rays; r0 += 32) {
        std::vector<Lane> L;
        for (size_t r = r0; r < std::min(n_rays, r0 + 32); ++r) {
            const float* R = &rays[8 * r];
            Lane l;
            for (int k = 0; k < 3; ++k) { l.o[k] = R[k]; l.d[k] = R[4 + k]; }
            l.tmin = R[3];
            l.best = R[7];
            l.oct = (l.d[0] >= 0 ? 1u : 0u) | (l.d[1] >= 0 ? 2u : 0u) | (l.d[2] >= 0 ? 4u : 0u);
            l.ng = {0u, (1u << (24 + l.oct)) | 1u};
            l.tg = {0u, 0u};
            l.bestp = -1;
            l.done = false;
            l.ray = r;
            L.push_back(l);
        }
        long steps = 0;
        for (;;) {
            bool any = false;
            for (Lane& l : L) any |= !l.done;
            if (!any) break;
            if (++steps > 1000000) return Fail("warp loop did not finish", (long)r0) ? 0 : 1;
            // Node step.
            for (Lane& l : L) {
                if (l.done) continue;
                l.tg = {0u, 0u};
                if (l.ng.second & 0xff000000u) {
                    const unsigned j = (unsigned)__builtin_ctz(l.ng.second >> 24);
                    l.ng.second &= ~(1u << (24 + j));
                    const unsigned slot = j ^ l.oct;
                    const uint32_t ni = l.ng.first + (uint32_t)__builtin_popcount(l.ng.second & 0xffu & ((1u << slot) - 1u));
                    if (l.ng.second & 0xff000000u) {
                        if ((int)l.stk.size() >= kStack) return Fail("stack overflow", (long)l.ray) ? 0 : 1;
                        l.stk.push_back(l.ng);
                    }
                    const WNode8& n = nodes[ni];
                    const float org[3] = {n.px, n.py, n.pz};
                    const int ex[3] = {n.ex, n.ey, n.ez};
                    const uint8_t* ql[3] = {n.qlox, n.qloy, n.qloz};
                    const uint8_t* qh[3] = {n.qhix, n.qhiy, n.qhiz};
                    uint32_t hn = 0, ht = 0;
                    for (int sl = 0; sl < 8; ++sl) {
                        double tn = l.tmin, tf = l.best;
                        for (int k = 0; k < 3; ++k) {
                            const double lo = Dec(org[k], ex[k], ql[k][sl]), hi = Dec(org[k], ex[k], qh[k][sl]);
                            if (l.d[k] == 0.0) {
                                if (l.o[k] < lo || l.o[k] > hi) tf = -1.0;
                                continue;
                            }
                            double a = (lo - l.o[k]) / l.d[k], c = (hi - l.o[k]) / l.d[k];
                            if (a > c) std::swap(a, c);
                            tn = std::fmax(tn, a);
                            tf = std::fmin(tf, c);
                        }
                        if (!(tn <= tf * (1 + 1e-9) + 1e-12)) continue;
                        if ((n.imask >> sl) & 1) hn |= 1u << (24 + (sl ^ l.oct));
                        else ht |= (uint32_t)(n.meta[sl] >> 5) << (n.meta[sl] & 31u);
                    }
                    l.ng = {n.child_base, hn | n.imask};
                    l.tg = {n.tri_base, ht};
                } else {
                    l.tg = l.ng;
                    l.ng = {0u, 0u};
                }
            }
            // Triangle loop in lockstep.
            std::vector<bool> inloop(L.size());
            for (size_t i = 0; i < L.size(); ++i) inloop[i] = !L[i].done && L[i].tg.second != 0;
            for (;;) {
                int count = 0;
                for (size_t i = 0; i < L.size(); ++i) count += inloop[i] ? 1 : 0;
                if (!count) break;
                for (size_t i = 0; i < L.size(); ++i) {
                    if (!inloop[i]) continue;
                    Lane& l = L[i];
                    if ((l.ng.second & 0xff000000u) && (int)l.stk.size() < kStack - kLevels && count < kTriLanes) {
                        l.stk.push_back(l.tg);
                        l.tg = {0u, 0u};
                        inloop[i] = false;
                        continue;
                    }
                    const unsigned k = (unsigned)__builtin_ctz(l.tg.second);
                    l.tg.second &= l.tg.second - 1;
                    const uint32_t p = prims[l.tg.first + k];
                    double t;
                    if (Hit(&tri9[9 * (size_t)p], l.o, l.d, t) && t > l.tmin && t < l.best) { l.best = t; l.bestp = (long)p; }
                    if (!l.tg.second) inloop[i] = false;
                }
            }
            for (Lane& l : L) {
                if (l.done || (l.ng.second & 0xff000000u)) continue;
                if (l.stk.empty()) { l.done = true; continue; }
                l.ng = l.stk.back();
                l.stk.pop_back();
            }
        }
        for (const Lane& l : L) {
            const float* R = &rays[8 * l.ray];
            const double o[3] = {R[0], R[1], R[2]}, d[3] = {R[4], R[5], R[6]};
            double bt = R[7];
            long best = -1;
            for (int64_t i = 0; i < n_tri; ++i) {
                double t;
                if (Hit(&tri9[9 * i], o, d, t) && t > R[3] && t < bt) { bt = t; best = (long)i; }
            }
            if (l.bestp != best && !(best >= 0 && l.bestp >= 0 && l.best == bt))
                return Fail("warp closest hit", (long)l.ray, l.bestp) ? 0 : 1;
        }
    }
    std::printf("ok %zu %d\n", nodes.size(), depth);
    return 0;
}
