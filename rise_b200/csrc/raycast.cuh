// raycast.cuh -- device-side BVH traversal and triangle tests for sm_100a.
//
// Shared by the batch ray-cast kernels (raycast.cu) and the wavefront path
// tracer (pathtrace.cu).  The traversal replaces the reference's single-ray
// BVH4 walk (src/Library/Acceleration/BVH.h:1304-1471) over the same
// collapsed tree with a warp-cooperative "while-while" walk: lanes first
// descend internal nodes until every lane holds a postponed leaf, then test
// leaves together, and a lane whose ray is finished takes the next ray from a
// warp-local chunk of the batch.  The reference's double-precision
// Moller-Trumbore leaf test (src/Library/Intersection/RayTriangleIntersection.cpp:21-68)
// becomes the FP32 watertight test of Woop, Benthin and Wald (JCGT 2(1), 2013);
// the closest hit is re-measured in FP64 with the reference's formula, so the
// reported distance is the reference's distance rounded once to FP32.
#pragma once
#include <climits>
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "bvh_build.h"

namespace rtb200 {

constexpr unsigned kErrStackOverflow = 1u;
constexpr int kEmpty = INT_MIN;      // no node / no leaf
constexpr int kTraceBlock = 128;     // threads per block of the trace kernels
// Traversal stack per thread: the first kTraceStack entries in shared memory
// (20 KB per block: 8 blocks of 128 threads stay resident per SM next to 64
// registers).  Kernels instantiated with SPILL continue it in local memory for
// scenes whose TraceStackBound exceeds kTraceStack; the others carry no local
// array at all.
constexpr int kTraceStack = kTraceStackShared;
constexpr int kTraceSpill = kTraceStackMax - kTraceStackShared;
constexpr unsigned kFull = 0xffffffffu;

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
        // Zero components map to FLT_MAX like the reference (BVH.h:1221-1224).
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
    const float adet = fabsf(det);
    // det is the Moller-Trumbore determinant e1 . (d x e2) divided by the
    // dominant direction component, |det_MT| = adet / |sz|: the reference
    // rejects |det_MT| < 1e-12 (RayTriangleIntersection.cpp:40-42), which
    // also drops triangles with edges below ~1e-6.
    if (!(adet >= 1e-12f * fabsf(p.sz))) return false;
    const float T = U * (p.sz * Az) + V * (p.sz * Bz) + W * (p.sz * Cz);
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
    int c[4];
    unsigned mask;
};

// Three-input minimum / maximum (one instruction on sm_100a).
__device__ __forceinline__ float Max3(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float Min3(float a, float b, float c)
{
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// FP32 node: the reference slab arithmetic (BVH.h:738-763) per child.  The
// reference takes min / max of the two plane distances per axis; with a
// finite reciprocal (zero components map to FLT_MAX) the near plane is the
// low one for a positive reciprocal and the high one otherwise, so loading
// the near and far planes by the ray's direction signs gives bit-identical
// entry / exit distances without the per-axis min / max.
__device__ __forceinline__ void SlabF32(const GpuNode4* nodes, int ni, const RayPre& p, float best, ChildHits& h)
{
    const float* base = reinterpret_cast<const float*>(nodes + ni);
    // Float offsets of lox, loy, loz, hix, hiy, hiz: 0, 4, 8, 12, 16, 20.
    const int nx = p.inv[0] < 0.0f ? 12 : 0, ny = p.inv[1] < 0.0f ? 16 : 4, nz = p.inv[2] < 0.0f ? 20 : 8;
    const float4 Nx = ldg4(base + nx), Ny = ldg4(base + ny), Nz = ldg4(base + nz);
    const float4 Fx = ldg4(base + (12 - nx)), Fy = ldg4(base + (20 - ny)), Fz = ldg4(base + (28 - nz));
    const int4 child = ldg4i(base + 24);   // empty slots hold kEmpty; counts are not read
    const float nxa[4] = {Nx.x, Nx.y, Nx.z, Nx.w}, nya[4] = {Ny.x, Ny.y, Ny.z, Ny.w}, nza[4] = {Nz.x, Nz.y, Nz.z, Nz.w};
    const float fxa[4] = {Fx.x, Fx.y, Fx.z, Fx.w}, fya[4] = {Fy.x, Fy.y, Fy.z, Fy.w}, fza[4] = {Fz.x, Fz.y, Fz.z, Fz.w};
    h.c[0] = child.x; h.c[1] = child.y; h.c[2] = child.z; h.c[3] = child.w;
    h.mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float tn = Max3((nxa[i] - p.o[0]) * p.inv[0], (nya[i] - p.o[1]) * p.inv[1],
                              fmaxf((nza[i] - p.o[2]) * p.inv[2], p.tmin));
        const float tf = Min3((fxa[i] - p.o[0]) * p.inv[0], (fya[i] - p.o[1]) * p.inv[1],
                              fminf((fza[i] - p.o[2]) * p.inv[2], best));
        h.t[i] = tn;
        if (tn <= tf && h.c[i] != kEmpty) h.mask |= 1u << i;
    }
}

// Quantised node: child slabs from 8-bit bounds, t = q * (2^e / d) + (origin - o) / d.
__device__ __forceinline__ void SlabQ8(const QNode4* nodes, int ni, const RayPre& p, float best, ChildHits& h)
{
    const int4* base = reinterpret_cast<const int4*>(nodes + ni);
    const int4 w0 = __ldg(base + 0), w1 = __ldg(base + 1), w2 = __ldg(base + 2), w3 = __ldg(base + 3);
    const float org[3] = {__int_as_float(w0.x), __int_as_float(w0.y), __int_as_float(w0.z)};
    const unsigned meta = (unsigned)w0.w;
    const int e[3] = {(int)(int8_t)(meta & 0xff), (int)(int8_t)((meta >> 8) & 0xff), (int)(int8_t)((meta >> 16) & 0xff)};
    // Near / far quantised planes per axis by the direction's sign (see SlabF32).
    const unsigned qlo[3] = {(unsigned)w1.x, (unsigned)w1.y, (unsigned)w1.z};
    const unsigned qhi[3] = {(unsigned)w1.w, (unsigned)w2.x, (unsigned)w2.y};
    unsigned qn[3], qf[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const bool neg = p.inv[k] < 0.0f;
        qn[k] = neg ? qhi[k] : qlo[k];
        qf[k] = neg ? qlo[k] : qhi[k];
    }
    h.c[0] = w2.z; h.c[1] = w2.w; h.c[2] = w3.x; h.c[3] = w3.y;
    const int cnt[4] = {(int)(int16_t)(w3.z & 0xffff), (int)(int16_t)((unsigned)w3.z >> 16),
                        (int)(int16_t)(w3.w & 0xffff), (int)(int16_t)((unsigned)w3.w >> 16)};
    float a[3], s[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a[k] = (org[k] - p.o[k]) * p.inv[k];
        s[k] = __int_as_float((e[k] + 127) << 23) * p.inv[k];
    }
    h.mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float tl[3], th[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            tl[k] = fmaf((float)((qn[k] >> (8 * i)) & 0xff), s[k], a[k]);
            th[k] = fmaf((float)((qf[k] >> (8 * i)) & 0xff), s[k], a[k]);
        }
        const float tn = Max3(tl[0], tl[1], fmaxf(tl[2], p.tmin));
        const float tf = Min3(th[0], th[1], fminf(th[2], best));
        h.t[i] = tn;
        if (tn <= tf && cnt[i] >= 0) h.mask |= 1u << i;
    }
}

// Half-precision node: the FP32 slab test on child boxes widened to binary16
// (outward), planes picked by the direction's sign as in SlabF32.
__device__ __forceinline__ float2 Halves(unsigned w)
{
    return __half22float2(*reinterpret_cast<const __half2*>(&w));
}
__device__ __forceinline__ void SlabF16(const HNode4* nodes, int ni, const RayPre& p, float best, ChildHits& h)
{
    const int4* base = reinterpret_cast<const int4*>(nodes + ni);
    const int4 w0 = __ldg(base + 0), w1 = __ldg(base + 1), w2 = __ldg(base + 2), w3 = __ldg(base + 3);
    // Words (two halves each): lo x, y, z then hi x, y, z, children 0-1 and 2-3.
    const unsigned lo[3][2] = {{(unsigned)w0.x, (unsigned)w0.y}, {(unsigned)w0.z, (unsigned)w0.w},
                               {(unsigned)w1.x, (unsigned)w1.y}};
    const unsigned hi[3][2] = {{(unsigned)w1.z, (unsigned)w1.w}, {(unsigned)w2.x, (unsigned)w2.y},
                               {(unsigned)w2.z, (unsigned)w2.w}};
    float tl[3][4], th[3][4];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const bool neg = p.inv[k] < 0.0f;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float2 n = Halves(neg ? hi[k][j] : lo[k][j]), f = Halves(neg ? lo[k][j] : hi[k][j]);
            tl[k][2 * j] = (n.x - p.o[k]) * p.inv[k];
            tl[k][2 * j + 1] = (n.y - p.o[k]) * p.inv[k];
            th[k][2 * j] = (f.x - p.o[k]) * p.inv[k];
            th[k][2 * j + 1] = (f.y - p.o[k]) * p.inv[k];
        }
    }
    h.c[0] = w3.x; h.c[1] = w3.y; h.c[2] = w3.z; h.c[3] = w3.w;
    h.mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float tn = Max3(tl[0][i], tl[1][i], fmaxf(tl[2][i], p.tmin));
        const float tf = Min3(th[0][i], th[1][i], fminf(th[2][i], best));
        h.t[i] = tn;
        if (tn <= tf && h.c[i] != kEmpty) h.mask |= 1u << i;
    }
}

template <class NodeT>
struct Slab;
template <>
struct Slab<GpuNode4> {
    __device__ __forceinline__ static void Run(const GpuNode4* n, int i, const RayPre& p, float b, ChildHits& h)
    {
        SlabF32(n, i, p, b, h);
    }
};
template <>
struct Slab<QNode4> {
    __device__ __forceinline__ static void Run(const QNode4* n, int i, const RayPre& p, float b, ChildHits& h)
    {
        SlabQ8(n, i, p, b, h);
    }
};
template <>
struct Slab<HNode4> {
    __device__ __forceinline__ static void Run(const HNode4* n, int i, const RayPre& p, float b, ChildHits& h)
    {
        SlabF16(n, i, p, b, h);
    }
};

__device__ __forceinline__ void CSwap(float& ta, int& ca, float& tb, int& cb)
{
    // After the call (ta, ca) holds the nearer entry.
    const bool sw = tb < ta;
    const float t = sw ? tb : ta;
    const int c = sw ? cb : ca;
    tb = sw ? ta : tb;
    cb = sw ? ca : cb;
    ta = t;
    ca = c;
}

// Per-lane traversal state of one ray.
struct TraceState {
    RayPre p;
    float d[3];        // direction (for the FP64 distance refinement)
    float best;        // current tmax
    int bestSlot;      // leaf-order triangle slot of the closest hit
    float ba, bb;      // its barycentrics
    int node;          // next internal node, a leaf entry (~first), or kEmpty
    int leaf;          // postponed leaf entry (~first) or kEmpty
    int sp;            // stack depth
};

__device__ __forceinline__ void StartRay(TraceState& s, const Ray& r)
{
    Prepare(r, s.p);
    s.d[0] = r.d[0]; s.d[1] = r.d[1]; s.d[2] = r.d[2];
    s.best = r.tmax;
    s.bestSlot = -1;
    s.ba = s.bb = 0.0f;
    s.node = 0;
    s.leaf = kEmpty;
    s.sp = 0;
}

// The stack: `stk` points at this thread's column of the shared-memory part
// ([depth][thread]); `spill` is the thread's local-memory continuation.
struct TraceStack {
    int* stk;
    int* spill;
};

// Overflow (a bound computed wrongly) drops the entry and raises the error
// flag, which the host turns into an error status.
template <bool SPILL>
__device__ __forceinline__ void Push(TraceState& s, const TraceStack& st, int v, unsigned* err)
{
    if (s.sp < kTraceStack) { st.stk[s.sp * kTraceBlock] = v; ++s.sp; }
    else if (SPILL && s.sp < kTraceStack + kTraceSpill) { st.spill[s.sp - kTraceStack] = v; ++s.sp; }
    else atomicOr(err, kErrStackOverflow);
}

template <bool SPILL>
__device__ __forceinline__ int Pop(TraceState& s, const TraceStack& st)
{
    if (s.sp == 0) return kEmpty;
    --s.sp;
    if (!SPILL || s.sp < kTraceStack) return st.stk[s.sp * kTraceBlock];
    return st.spill[s.sp - kTraceStack];
}

// Lanes of a warp that may still lack a postponed leaf when the descent
// stops: waiting for the last few lanes to find one left most lanes idle.
constexpr int kDescentLanes = 12;

// One round of while-while traversal for every active lane: descend internal
// nodes until fewer than kDescentLanes active lanes still lack a postponed
// leaf (or have run out of nodes), then test at most LEAVES leaves per lane
// as one flat walk over their triangles; a leaf met after that is kept for the
// next round, whose descent starts with it.  Measured on incoherent rays
// (4-wide nodes, where sibling leaves are common): with uncapped leaf chains
// and a descent that waited for every lane, 25 % of the lanes were active in
// the leaf loop and 42 % in the descent; the cap, the flat walk and the early
// stop together trace 70 % more rays per second.  ANY: stop at the first
// accepted hit.  Returns true when this lane's ray is finished.
template <class NodeT, bool ANY, bool SPILL, int LEAVES>
__device__ __forceinline__ bool TraceRound(TraceState& s, const NodeT* __restrict__ nodes,
                                           const GpuTri* __restrict__ tris, int ntri, const TraceStack& stk, unsigned* err)
{
    // Descend internal nodes, first postponing a leaf left from the last round.
    for (;;) {
        if (s.node < 0 && s.node != kEmpty && s.leaf == kEmpty) {
            s.leaf = s.node;
            s.node = Pop<SPILL>(s, stk);
        }
        if (s.node < 0) break;
        ChildHits h;
        Slab<NodeT>::Run(nodes, s.node, s.p, s.best, h);
        // Nearest-first ordering of the (up to 4) hit children.
        float t0 = (h.mask & 1u) ? h.t[0] : __int_as_float(0x7f800000);
        float t1 = (h.mask & 2u) ? h.t[1] : __int_as_float(0x7f800000);
        float t2 = (h.mask & 4u) ? h.t[2] : __int_as_float(0x7f800000);
        float t3 = (h.mask & 8u) ? h.t[3] : __int_as_float(0x7f800000);
        int c0 = (h.mask & 1u) ? h.c[0] : kEmpty;
        int c1 = (h.mask & 2u) ? h.c[1] : kEmpty;
        int c2 = (h.mask & 4u) ? h.c[2] : kEmpty;
        int c3 = (h.mask & 8u) ? h.c[3] : kEmpty;
        CSwap(t0, c0, t1, c1);
        CSwap(t2, c2, t3, c3);
        CSwap(t0, c0, t2, c2);
        CSwap(t1, c1, t3, c3);
        CSwap(t1, c1, t2, c2);
        // Push far to near; the nearest becomes the next node.
        if (c3 != kEmpty) Push<SPILL>(s, stk, c3, err);
        if (c2 != kEmpty) Push<SPILL>(s, stk, c2, err);
        if (c1 != kEmpty) Push<SPILL>(s, stk, c1, err);
        s.node = (c0 != kEmpty) ? c0 : Pop<SPILL>(s, stk);
        // Postpone the first leaf met; keep descending until most lanes have one.
        if (s.node < 0 && s.node != kEmpty && s.leaf == kEmpty) {
            s.leaf = s.node;
            s.node = Pop<SPILL>(s, stk);
        }
        if (__popc(__ballot_sync(__activemask(), s.leaf == kEmpty)) < kDescentLanes) break;
    }
    // Test leaves: one walk over the triangles of up to LEAVES leaves.
    int nleaf = 0;
    int slot = s.leaf != kEmpty ? ~s.leaf : -1;
    while (slot >= 0) {
        const float* tb = reinterpret_cast<const float*>(tris + slot);
        const float4 A = ldg4(tb), B = ldg4(tb + 4), C = ldg4(tb + 8);
        float t, a, b;
        if (Watertight(s.p, A, B, C, s.best, t, a, b)) {
            if (ANY) {
                s.bestSlot = slot;
                s.node = kEmpty;
                s.leaf = kEmpty;
                return true;
            }
            s.best = t;
            s.bestSlot = slot;
            s.ba = a;
            s.bb = b;
        }
        // The last triangle of a leaf carries v1.w = 1; the array bound is a
        // second stop so a leaf walk never leaves the buffer.
        if (B.w != 0.0f || slot + 1 >= ntri) {
            s.leaf = kEmpty;
            slot = -1;
            if (++nleaf < LEAVES && s.node < 0 && s.node != kEmpty) {
                s.leaf = s.node;
                s.node = Pop<SPILL>(s, stk);
                slot = ~s.leaf;
            }
        } else {
            ++slot;
        }
    }
    return s.node == kEmpty && s.leaf == kEmpty;
}

// ---- eight-wide compressed nodes (WNode8, bvh_wide.cpp) -------------------
// Per-lane traversal after Ylitie, Karras and Laine (HPG 2017): a node group
// (first internal child's index; hit children in bits 24-31 in visiting
// order, the node's internal-child mask in bits 0-7) and a triangle group
// (first triangle; hit triangles in bits 0-23).  A node's hit children are
// visited in slot order s ^ oct, oct the ray's non-negative direction signs,
// which the build made roughly near to far; groups wait on a stack of one
// entry per tree level, bounded at commit.

constexpr int kW8Stack = kW8StackEntries;   // uint2 entries per thread in shared memory
constexpr int kW8Levels = kW8MaxLevels;      // node groups the stack keeps room for

struct W8State {
    RayPre p;
    float d[3];
    float best;
    int bestSlot;
    float ba, bb;
    unsigned oct;
    uint2 ng;          // node group
    int sp;
    int visits;        // iterations spent on this ray (bounded)
};

// A ray takes at most this many iterations (each visits one node or tests
// one triangle group; a tree of n triangles has fewer than n nodes), else its
// traversal stops with the error flag raised.
constexpr int kW8MaxIterations = 1 << 22;

__device__ __forceinline__ void StartRayW8(W8State& s, const Ray& r)
{
    Prepare(r, s.p);
    s.d[0] = r.d[0]; s.d[1] = r.d[1]; s.d[2] = r.d[2];
    s.best = r.tmax;
    s.bestSlot = -1;
    s.ba = s.bb = 0.0f;
    s.oct = (r.d[0] >= 0.0f ? 1u : 0u) | (r.d[1] >= 0.0f ? 2u : 0u) | (r.d[2] >= 0.0f ? 4u : 0u);
    // The root as the one internal child (slot 0) of a virtual parent at 0.
    s.ng = make_uint2(0u, (1u << (24 + s.oct)) | 1u);
    s.sp = 0;
    s.visits = 0;
}

// Child slabs of one node: the node group of its hit internal children and
// the triangle group of its hit leaf slots.
__device__ __forceinline__ void IntersectW8(const WNode8* __restrict__ nodes, unsigned ni, const RayPre& p,
                                            unsigned oct, float best, uint2& ng, uint2& tg)
{
    const uint4* base = reinterpret_cast<const uint4*>(nodes + ni);
    const uint4 w0 = __ldg(base), w1 = __ldg(base + 1), w2 = __ldg(base + 2), w3 = __ldg(base + 3),
                w4 = __ldg(base + 4);
    const float org[3] = {__uint_as_float(w0.x), __uint_as_float(w0.y), __uint_as_float(w0.z)};
    const unsigned em = w0.w;
    const int e[3] = {(int)(int8_t)(em & 0xffu), (int)(int8_t)((em >> 8) & 0xffu), (int)(int8_t)((em >> 16) & 0xffu)};
    const unsigned imask = em >> 24;
    // Bounds per axis as two words of four bytes (slots 0-3, 4-7); near and
    // far planes by the direction's sign (see SlabF32).
    const unsigned lo[3][2] = {{w2.x, w2.y}, {w2.z, w2.w}, {w3.x, w3.y}};
    const unsigned hi[3][2] = {{w3.z, w3.w}, {w4.x, w4.y}, {w4.z, w4.w}};
    unsigned qn[3][2], qf[3][2];
    float a[3], sc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const bool neg = p.inv[k] < 0.0f;
        qn[k][0] = neg ? hi[k][0] : lo[k][0];
        qn[k][1] = neg ? hi[k][1] : lo[k][1];
        qf[k][0] = neg ? lo[k][0] : hi[k][0];
        qf[k][1] = neg ? lo[k][1] : hi[k][1];
        a[k] = (org[k] - p.o[k]) * p.inv[k];
        sc[k] = __int_as_float((e[k] + 127) << 23) * p.inv[k];
    }
    unsigned hitsN = 0u, hitsT = 0u;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int h = i >> 2, sh = 8 * (i & 3);
        float tl[3], th[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            tl[k] = fmaf((float)((qn[k][h] >> sh) & 0xffu), sc[k], a[k]);
            th[k] = fmaf((float)((qf[k][h] >> sh) & 0xffu), sc[k], a[k]);
        }
        const float tn = Max3(tl[0], tl[1], fmaxf(tl[2], p.tmin));
        const float tf = Min3(th[0], th[1], fminf(th[2], best));
        if (tn <= tf) {
            if ((imask >> i) & 1u) {
                hitsN |= 1u << (24 + (i ^ oct));
            } else {
                const unsigned meta = ((i < 4 ? w1.z : w1.w) >> sh) & 0xffu;
                hitsT |= (meta >> 5) << (meta & 31u);
            }
        }
    }
    ng = make_uint2(w1.x, hitsN | imask);
    tg = make_uint2(w1.y, hitsT);
}

// Lanes below which a warp postpones its triangle tests (pushes the
// triangle group and keeps descending), after Ylitie et al.
constexpr int kW8TriLanes = 8;

// Traverses for at most `budget` iterations; returns true when the ray is
// finished.  The current group `ng` is a node group (hits in bits 24-31) or,
// popped from the stack, a postponed triangle group (bits 0-23 only).  A
// triangle group is postponed while fewer than kW8TriLanes lanes of the warp
// have triangles to test and the stack keeps room for one node group per
// level (kW8Levels).  ANY: stop at the first accepted hit.
template <bool ANY>
__device__ __forceinline__ bool TraceW8(W8State& s, const WNode8* __restrict__ nodes,
                                        const GpuTri* __restrict__ tris, uint2* stk, unsigned* err, int budget)
{
    for (int it = 0; it < budget; ++it) {
        if (++s.visits > kW8MaxIterations) {
            atomicOr(err, kErrStackOverflow);
            return true;
        }
        uint2 tg = make_uint2(0u, 0u);
        if (s.ng.y & 0xff000000u) {
            const unsigned j = (unsigned)__ffs(s.ng.y >> 24) - 1u;
            s.ng.y &= ~(1u << (24 + j));
            const unsigned slot = j ^ s.oct;
            const unsigned ni = s.ng.x + (unsigned)__popc(s.ng.y & 0xffu & ((1u << slot) - 1u));
            if (s.ng.y & 0xff000000u) {
                if (s.sp < kW8Stack) { stk[s.sp * kTraceBlock] = s.ng; ++s.sp; }
                else atomicOr(err, kErrStackOverflow);
            }
            IntersectW8(nodes, ni, s.p, s.oct, s.best, s.ng, tg);
        } else {
            tg = s.ng;   // a postponed triangle group (or nothing)
            s.ng = make_uint2(0u, 0u);
        }
        while (tg.y) {
            // Postpone only with a node group to continue with, so a popped
            // triangle group is always tested (the ray keeps progressing).
            if ((s.ng.y & 0xff000000u) && s.sp < kW8Stack - kW8Levels &&
                __popc(__ballot_sync(__activemask(), true)) < kW8TriLanes) {
                stk[s.sp * kTraceBlock] = tg;
                ++s.sp;
                break;
            }
            const unsigned k = (unsigned)__ffs(tg.y) - 1u;
            tg.y &= tg.y - 1u;
            const unsigned slot = tg.x + k;
            const float* tb = reinterpret_cast<const float*>(tris + slot);
            const float4 A = ldg4(tb), B = ldg4(tb + 4), C = ldg4(tb + 8);
            float t, al, be;
            if (Watertight(s.p, A, B, C, s.best, t, al, be)) {
                s.bestSlot = (int)slot;
                if (ANY) return true;
                s.best = t;
                s.ba = al;
                s.bb = be;
            }
        }
        if (!(s.ng.y & 0xff000000u)) {
            if (s.sp == 0) return true;
            --s.sp;
            s.ng = stk[s.sp * kTraceBlock];
        }
    }
    return false;
}

// Warp-cooperative ray supply: a lane whose ray is finished takes the next
// index from a warp-local chunk; the chunk is refilled from the global
// counter kChunk rays at a time (one atomic per chunk per warp).
struct WarpFeed {
    unsigned long long next, end;
    bool exhausted;
};

constexpr unsigned kChunk = 128;

// Returns this lane's new ray index or -1.  `want` lanes ask for work.
__device__ __forceinline__ long long FeedTake(WarpFeed& f, bool want, unsigned long long n,
                                              unsigned long long* counter)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned wm = __ballot_sync(kFull, want);
    if (!wm) return -1;
    const unsigned need = __popc(wm);
    const unsigned rank = __popc(wm & ((1u << lane) - 1u));
    unsigned long long avail = f.end - f.next;
    long long mine = -1;
    if (rank < avail) mine = (long long)(f.next + rank);
    if (avail < need && !f.exhausted) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, (unsigned long long)kChunk);
        base = __shfl_sync(kFull, base, 0);
        if (base >= n) {
            f.exhausted = true;
            f.next = f.end;
        } else {
            const unsigned long long end = (base + kChunk < n) ? base + kChunk : n;
            const unsigned long long extra = need - avail;
            if (rank >= avail && base + (rank - avail) < end) mine = (long long)(base + (rank - avail));
            f.next = (base + extra < end) ? base + extra : end;
            f.end = end;
            if (end == n) f.exhausted = true;
        }
    } else {
        f.next += (avail < need) ? avail : need;
    }
    return want ? mine : -1;
}

}  // namespace rtb200
