// raycast.cuh -- device-side BVH traversal and triangle tests for sm_100a.
//
// Shared by the batch ray-cast kernels (raycast.cu) and the wavefront path
// tracer (pathtrace.cu).  The traversal replaces the reference's single-ray
// BVH4 walk (src/Library/Acceleration/BVH.h:1304-1471) with a per-thread
// stack walk over the same collapsed tree, and the reference's
// double-precision Moller-Trumbore leaf test
// (src/Library/Intersection/RayTriangleIntersection.cpp:21-68) with the FP32
// watertight test of Woop, Benthin and Wald (JCGT 2(1), 2013).  The closest hit
// is re-measured in FP64 with the reference's formula, so the reported distance
// is the reference's distance rounded once to FP32.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "bvh_build.h"

namespace rtb200 {

constexpr int kStackSize = 96;
constexpr unsigned kErrStackOverflow = 1u;

struct Ray {
    float o[3];
    float tmin;
    float d[3];
    float tmax;
};

struct RayPre {
    float o[3];
    float inv[3];
    float tmin;
    // watertight shear
    int kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ float4 ldg4(const void* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ int4 ldg4i(const void* p) { return __ldg(reinterpret_cast<const int4*>(p)); }

__device__ __forceinline__ float Comp(const float* v, int k) { return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]); }

__device__ __forceinline__ void Prepare(const Ray& r, RayPre& p)
{
    for (int k = 0; k < 3; ++k) {
        p.o[k] = r.o[k];
        // Zero components map to +-FLT_MAX like the reference (BVH.h:1221-1224).
        p.inv[k] = (r.d[k] == 0.0f) ? 3.402823466e+38f : __frcp_rn(r.d[k]);
    }
    p.tmin = r.tmin;
    const float ax = fabsf(r.d[0]), ay = fabsf(r.d[1]), az = fabsf(r.d[2]);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    const float dz = Comp(r.d, kz);
    if (dz < 0.0f) { int t = kx; kx = ky; ky = t; }
    p.kx = kx; p.ky = ky; p.kz = kz;
    p.sx = Comp(r.d, kx) / dz;
    p.sy = Comp(r.d, ky) / dz;
    p.sz = 1.0f / dz;
}

// Watertight ray/triangle test.  Returns true for a hit with tmin < t < tmax
// and writes t and the barycentrics (alpha, beta) of v1 and v2, the
// reference's (a, b) convention.
__device__ __forceinline__ bool Watertight(const RayPre& p, const float4& A4, const float4& B4,
                                           const float4& C4, float tmax, float& tOut, float& aOut,
                                           float& bOut)
{
    const float A[3] = {A4.x - p.o[0], A4.y - p.o[1], A4.z - p.o[2]};
    const float B[3] = {B4.x - p.o[0], B4.y - p.o[1], B4.z - p.o[2]};
    const float C[3] = {C4.x - p.o[0], C4.y - p.o[1], C4.z - p.o[2]};
    const float Az = Comp(A, p.kz), Bz = Comp(B, p.kz), Cz = Comp(C, p.kz);
    const float Ax = Comp(A, p.kx) - p.sx * Az, Ay = Comp(A, p.ky) - p.sy * Az;
    const float Bx = Comp(B, p.kx) - p.sx * Bz, By = Comp(B, p.ky) - p.sy * Bz;
    const float Cx = Comp(C, p.kx) - p.sx * Cz, Cy = Comp(C, p.ky) - p.sy * Cz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        // Edge case: redo the 2D edge functions in FP64 (paper, section 3).
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float T = U * (p.sz * Az) + V * (p.sz * Bz) + W * (p.sz * Cz);
    const float adet = fabsf(det);
    const float sT = copysignf(1.0f, det) * T;
    if (sT <= p.tmin * adet || sT >= tmax * adet) return false;
    const float rcp = 1.0f / det;
    tOut = T * rcp;
    aOut = V * rcp;
    bOut = W * rcp;
    return true;
}

// The reference's double-precision Moller-Trumbore distance for a triangle
// already known to be hit (RayTriangleIntersection.cpp:36-60).
__device__ __forceinline__ double RefineT(const float* o, const float* d, const float4& A4,
                                          const float4& B4, const float4& C4)
{
    const double ea[3] = {(double)B4.x - A4.x, (double)B4.y - A4.y, (double)B4.z - A4.z};
    const double eb[3] = {(double)C4.x - A4.x, (double)C4.y - A4.y, (double)C4.z - A4.z};
    const double dd[3] = {d[0], d[1], d[2]};
    const double pv[3] = {dd[1] * eb[2] - dd[2] * eb[1], dd[2] * eb[0] - dd[0] * eb[2], dd[0] * eb[1] - dd[1] * eb[0]};
    const double det = ea[0] * pv[0] + ea[1] * pv[1] + ea[2] * pv[2];
    const double tv[3] = {(double)o[0] - A4.x, (double)o[1] - A4.y, (double)o[2] - A4.z};
    const double qv[3] = {tv[1] * ea[2] - tv[2] * ea[1], tv[2] * ea[0] - tv[0] * ea[2], tv[0] * ea[1] - tv[1] * ea[0]};
    return (eb[0] * qv[0] + eb[1] * qv[1] + eb[2] * qv[2]) / det;
}

// ---- node decoders --------------------------------------------------------

struct ChildHits {
    float t[4];
    unsigned mask;
};

// FP32 node: the reference slab arithmetic (BVH.h:738-763) per child.
__device__ __forceinline__ void SlabF32(const GpuNode4* nodes, int ni, const RayPre& p, float best,
                                        ChildHits& h, int4& child, int4& count)
{
    const float* base = reinterpret_cast<const float*>(nodes + ni);
    const float4 lx = ldg4(base + 0), ly = ldg4(base + 4), lz = ldg4(base + 8);
    const float4 hx = ldg4(base + 12), hy = ldg4(base + 16), hz = ldg4(base + 20);
    child = ldg4i(base + 24);
    count = ldg4i(base + 28);
    const float lxa[4] = {lx.x, lx.y, lx.z, lx.w}, lya[4] = {ly.x, ly.y, ly.z, ly.w}, lza[4] = {lz.x, lz.y, lz.z, lz.w};
    const float hxa[4] = {hx.x, hx.y, hx.z, hx.w}, hya[4] = {hy.x, hy.y, hy.z, hy.w}, hza[4] = {hz.x, hz.y, hz.z, hz.w};
    const int cnt[4] = {count.x, count.y, count.z, count.w};
    h.mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float t1x = (lxa[i] - p.o[0]) * p.inv[0], t2x = (hxa[i] - p.o[0]) * p.inv[0];
        const float t1y = (lya[i] - p.o[1]) * p.inv[1], t2y = (hya[i] - p.o[1]) * p.inv[1];
        const float t1z = (lza[i] - p.o[2]) * p.inv[2], t2z = (hza[i] - p.o[2]) * p.inv[2];
        float tn = fmaxf(fmaxf(fminf(t1x, t2x), fminf(t1y, t2y)), fminf(t1z, t2z));
        float tf = fminf(fminf(fmaxf(t1x, t2x), fmaxf(t1y, t2y)), fmaxf(t1z, t2z));
        tn = fmaxf(tn, p.tmin);
        tf = fminf(tf, best);
        h.t[i] = tn;
        if (tn <= tf && cnt[i] >= 0) h.mask |= 1u << i;
    }
}

// Quantised node: child slabs from 8-bit bounds, t = q * (2^e / d) + (origin - o) / d.
__device__ __forceinline__ void SlabQ8(const QNode4* nodes, int ni, const RayPre& p, float best,
                                       ChildHits& h, int4& child, int4& count)
{
    const int4* base = reinterpret_cast<const int4*>(nodes + ni);
    const int4 w0 = __ldg(base + 0), w1 = __ldg(base + 1), w2 = __ldg(base + 2), w3 = __ldg(base + 3);
    const float org[3] = {__int_as_float(w0.x), __int_as_float(w0.y), __int_as_float(w0.z)};
    const unsigned meta = (unsigned)w0.w;
    const int e[3] = {(int)(int8_t)(meta & 0xff), (int)(int8_t)((meta >> 8) & 0xff), (int)(int8_t)((meta >> 16) & 0xff)};
    const unsigned qlo[3] = {(unsigned)w1.x, (unsigned)w1.y, (unsigned)w1.z};
    const unsigned qhi[3] = {(unsigned)w1.w, (unsigned)w2.x, (unsigned)w2.y};
    child = make_int4(w2.z, w2.w, w3.x, w3.y);
    count = make_int4((int)(int16_t)(w3.z & 0xffff), (int)(int16_t)((unsigned)w3.z >> 16),
                      (int)(int16_t)(w3.w & 0xffff), (int)(int16_t)((unsigned)w3.w >> 16));
    float a[3], s[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a[k] = (org[k] - p.o[k]) * p.inv[k];
        s[k] = __int_as_float((e[k] + 127) << 23) * p.inv[k];
    }
    const int cnt[4] = {count.x, count.y, count.z, count.w};
    h.mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float tl[3], th[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float ql = (float)((qlo[k] >> (8 * i)) & 0xff);
            const float qh = (float)((qhi[k] >> (8 * i)) & 0xff);
            const float t1 = fmaf(ql, s[k], a[k]);
            const float t2 = fmaf(qh, s[k], a[k]);
            tl[k] = fminf(t1, t2);
            th[k] = fmaxf(t1, t2);
        }
        float tn = fmaxf(fmaxf(fmaxf(tl[0], tl[1]), tl[2]), p.tmin);
        float tf = fminf(fminf(fminf(th[0], th[1]), th[2]), best);
        h.t[i] = tn;
        if (tn <= tf && cnt[i] >= 0) h.mask |= 1u << i;
    }
}

template <class NodeT>
struct Slab;
template <>
struct Slab<GpuNode4> {
    __device__ __forceinline__ static void Run(const GpuNode4* n, int i, const RayPre& p, float b, ChildHits& h, int4& c, int4& k)
    {
        SlabF32(n, i, p, b, h, c, k);
    }
};
template <>
struct Slab<QNode4> {
    __device__ __forceinline__ static void Run(const QNode4* n, int i, const RayPre& p, float b, ChildHits& h, int4& c, int4& k)
    {
        SlabQ8(n, i, p, b, h, c, k);
    }
};

__device__ __forceinline__ int Sel(const int4& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }

struct HitRecord {
    float t;
    int prim;     // leaf-order triangle slot, -1 = miss
    float a, b;
};

// Closest hit.  Returns the leaf-order slot of the closest triangle.
template <class NodeT>
__device__ __forceinline__ HitRecord TraceClosest(const NodeT* __restrict__ nodes, const GpuTri* __restrict__ tris,
                                                  const Ray& r, unsigned* err)
{
    RayPre p;
    Prepare(r, p);
    HitRecord hit;
    hit.t = r.tmax;
    hit.prim = -1;
    hit.a = hit.b = 0.0f;
    int stack[kStackSize];
    int sp = 0;
    int node = 0;
    for (;;) {
        ChildHits h;
        int4 child, count;
        Slab<NodeT>::Run(nodes, node, p, hit.t, h, child, count);
        // Leaves first, in slot order.
        unsigned inner = 0;
        unsigned m = h.mask;
        while (m) {
            const int i = __ffs(m) - 1;
            m &= m - 1;
            const int c = Sel(count, i);
            if (c > 0) {
                const int first = Sel(child, i);
                for (int s = first; s < first + c; ++s) {
                    const float* tb = reinterpret_cast<const float*>(tris + s);
                    const float4 A = ldg4(tb), B = ldg4(tb + 4), C = ldg4(tb + 8);
                    float t, a, b;
                    if (Watertight(p, A, B, C, hit.t, t, a, b)) {
                        hit.t = t; hit.prim = s; hit.a = a; hit.b = b;
                    }
                }
            } else {
                inner |= 1u << i;
            }
        }
        // Internal children: continue with the nearest, push the rest far-first.
        int next = -1;
        if (inner) {
            int ord[4];
            float key[4];
            int n = 0;
            while (inner) {
                const int i = __ffs(inner) - 1;
                inner &= inner - 1;
                ord[n] = Sel(child, i);
                key[n] = h.t[i];
                ++n;
            }
            // Sort descending by entry distance (n <= 4).
            for (int x = 1; x < n; ++x) {
                const float kk = key[x];
                const int oo = ord[x];
                int y = x - 1;
                while (y >= 0 && key[y] < kk) { key[y + 1] = key[y]; ord[y + 1] = ord[y]; --y; }
                key[y + 1] = kk;
                ord[y + 1] = oo;
            }
            for (int x = 0; x < n - 1; ++x) {
                if (sp < kStackSize) stack[sp++] = ord[x];
                else atomicOr(err, kErrStackOverflow);
            }
            next = ord[n - 1];
        }
        if (next < 0) {
            if (sp == 0) break;
            next = stack[--sp];
        }
        node = next;
    }
    return hit;
}

// Any hit within (tmin, tmax): returns true at the first accepted triangle.
template <class NodeT>
__device__ __forceinline__ bool TraceAny(const NodeT* __restrict__ nodes, const GpuTri* __restrict__ tris,
                                         const Ray& r, unsigned* err)
{
    RayPre p;
    Prepare(r, p);
    int stack[kStackSize];
    int sp = 0;
    int node = 0;
    for (;;) {
        ChildHits h;
        int4 child, count;
        Slab<NodeT>::Run(nodes, node, p, r.tmax, h, child, count);
        int next = -1;
        unsigned m = h.mask;
        while (m) {
            const int i = __ffs(m) - 1;
            m &= m - 1;
            const int c = Sel(count, i);
            const int first = Sel(child, i);
            if (c > 0) {
                for (int s = first; s < first + c; ++s) {
                    const float* tb = reinterpret_cast<const float*>(tris + s);
                    const float4 A = ldg4(tb), B = ldg4(tb + 4), C = ldg4(tb + 8);
                    float t, a, b;
                    if (Watertight(p, A, B, C, r.tmax, t, a, b)) return true;
                }
            } else if (next < 0) {
                next = first;
            } else if (sp < kStackSize) {
                stack[sp++] = first;
            } else {
                atomicOr(err, kErrStackOverflow);
            }
        }
        if (next < 0) {
            if (sp == 0) return false;
            next = stack[--sp];
        }
        node = next;
    }
}

}  // namespace rtb200
