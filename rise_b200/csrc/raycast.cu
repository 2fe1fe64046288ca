// raycast.cu -- batched closest-hit and any-hit kernels for sm_100a.
//
// Persistent kernels: one grid of (SMs x resident blocks); each warp takes
// 32 rays at a time from a per-scene work counter in global memory, so warps
// whose rays finish early pick up more work instead of idling while the
// slowest rays of a static partition finish.  Rays are read as two 16-byte
// vector loads and hits written as one 16-byte store.
#include "core.h"
#include "raycast.cuh"

namespace rtb200 {

constexpr int kCastBlock = 256;

template <class NodeT>
__global__ void __launch_bounds__(kCastBlock)
KCastClosest(const NodeT* __restrict__ nodes, const GpuTri* __restrict__ tris,
             const rtb200_ray* __restrict__ rays, int64_t n, rtb200_hit* __restrict__ hits,
             unsigned long long* counter, unsigned* err)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)n) return;
        const int64_t i = (int64_t)base + lane;
        if (i < n) {
            const float4 a = ldg4(rays + i);
            const float4 b = ldg4(reinterpret_cast<const float*>(rays + i) + 4);
            Ray r;
            r.o[0] = a.x; r.o[1] = a.y; r.o[2] = a.z; r.tmin = a.w;
            r.d[0] = b.x; r.d[1] = b.y; r.d[2] = b.z; r.tmax = b.w;
            const HitRecord h = TraceClosest<NodeT>(nodes, tris, r, err);
            float4 out;
            if (h.prim >= 0) {
                const float* tb = reinterpret_cast<const float*>(tris + h.prim);
                const float4 A = ldg4(tb), B = ldg4(tb + 4), C = ldg4(tb + 8);
                out.x = (float)RefineT(r.o, r.d, A, B, C);
                out.y = A.w;  // input triangle index (bit pattern)
                out.z = h.a;
                out.w = h.b;
            } else {
                out.x = -1.0f;
                out.y = __int_as_float(-1);
                out.z = 0.0f;
                out.w = 0.0f;
            }
            *reinterpret_cast<float4*>(hits + i) = out;
        }
    }
}

template <class NodeT>
__global__ void __launch_bounds__(kCastBlock)
KCastAny(const NodeT* __restrict__ nodes, const GpuTri* __restrict__ tris,
         const rtb200_ray* __restrict__ rays, int64_t n, uint8_t* __restrict__ occ,
         unsigned long long* counter, unsigned* err)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)n) return;
        const int64_t i = (int64_t)base + lane;
        if (i < n) {
            const float4 a = ldg4(rays + i);
            const float4 b = ldg4(reinterpret_cast<const float*>(rays + i) + 4);
            Ray r;
            r.o[0] = a.x; r.o[1] = a.y; r.o[2] = a.z; r.tmin = a.w;
            r.d[0] = b.x; r.d[1] = b.y; r.d[2] = b.z; r.tmax = b.w;
            occ[i] = TraceAny<NodeT>(nodes, tris, r, err) ? 1 : 0;
        }
    }
}

namespace {

template <class K>
int GridFor(K kernel, int num_sms)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kCastBlock, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * num_sms;
}

}  // namespace

cudaError_t LaunchCastClosest(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                              rtb200_hit* d_hits, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(s->d_counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    if (s->layout == RTB200_BVH_Q8) {
        static int grid = 0;
        if (!grid) grid = GridFor(KCastClosest<QNode4>, s->ctx->num_sms);
        KCastClosest<QNode4><<<grid, kCastBlock, 0, stream>>>((const QNode4*)s->d_nodes, s->d_tris, d_rays, n,
                                                              d_hits, s->d_counter, s->d_err);
    } else {
        static int grid = 0;
        if (!grid) grid = GridFor(KCastClosest<GpuNode4>, s->ctx->num_sms);
        KCastClosest<GpuNode4><<<grid, kCastBlock, 0, stream>>>((const GpuNode4*)s->d_nodes, s->d_tris, d_rays,
                                                                n, d_hits, s->d_counter, s->d_err);
    }
    return cudaGetLastError();
}

cudaError_t LaunchCastAny(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                          uint8_t* d_occ, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(s->d_counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    if (s->layout == RTB200_BVH_Q8) {
        static int grid = 0;
        if (!grid) grid = GridFor(KCastAny<QNode4>, s->ctx->num_sms);
        KCastAny<QNode4><<<grid, kCastBlock, 0, stream>>>((const QNode4*)s->d_nodes, s->d_tris, d_rays, n, d_occ,
                                                          s->d_counter, s->d_err);
    } else {
        static int grid = 0;
        if (!grid) grid = GridFor(KCastAny<GpuNode4>, s->ctx->num_sms);
        KCastAny<GpuNode4><<<grid, kCastBlock, 0, stream>>>((const GpuNode4*)s->d_nodes, s->d_tris, d_rays, n,
                                                            d_occ, s->d_counter, s->d_err);
    }
    return cudaGetLastError();
}

}  // namespace rtb200
