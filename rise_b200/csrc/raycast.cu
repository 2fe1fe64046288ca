// raycast.cu -- batched closest-hit and any-hit kernels for sm_100a.
//
// Persistent kernels: one grid of (SMs x resident blocks).  Each warp runs the
// while-while traversal of raycast.cuh; lanes refill themselves with new rays
// from a warp-local chunk as soon as their ray finishes, so SIMT lanes stay
// busy on the long tail of incoherent rays.  Rays are read as two 16-byte
// vector loads and hits written as one 16-byte store; the traversal stack
// lives in shared memory ([depth][thread], conflict-free).
#include <atomic>

#include "core.h"
#include "raycast.cuh"

namespace rtb200 {

__device__ __forceinline__ Ray LoadRay(const rtb200_ray* rays, long long i)
{
    const float4 a = ldg4(rays + i);
    const float4 b = ldg4(reinterpret_cast<const float*>(rays + i) + 4);
    Ray r;
    r.o[0] = a.x; r.o[1] = a.y; r.o[2] = a.z; r.tmin = a.w;
    r.d[0] = b.x; r.d[1] = b.y; r.d[2] = b.z; r.tmax = b.w;
    return r;
}

// Leaves tested per lane per traversal round in the batch kernels (measured
// best for both closest and any hit on incoherent rays).
constexpr int kCastLeaves = 2;

template <class NodeT, bool ANY, bool SPILL>
__global__ void __launch_bounds__(kTraceBlock, 8)
KTrace(const NodeT* __restrict__ nodes, const GpuTri* __restrict__ tris,
       const rtb200_ray* __restrict__ rays, long long n, int ntri, rtb200_hit* __restrict__ hits,
       uint8_t* __restrict__ occ, unsigned long long* counter, unsigned* err)
{
    __shared__ int sstack[kTraceStack * kTraceBlock];
    int spill[SPILL ? kTraceSpill : 1];
    const TraceStack stk{sstack + threadIdx.x, spill};
    WarpFeed feed{0ull, 0ull, false};
    TraceState s;
    long long ray = -1;
    for (;;) {
        const long long got = FeedTake(feed, ray < 0, (unsigned long long)n, counter);
        if (got >= 0) {
            ray = got;
            StartRay(s, LoadRay(rays, ray));
        }
        if (__all_sync(kFull, ray < 0)) break;
        if (ray >= 0 && TraceRound<NodeT, ANY, SPILL, kCastLeaves>(s, nodes, tris, ntri, stk, err)) {
            if (ANY) {
                occ[ray] = s.bestSlot >= 0 ? 1 : 0;
            } else {
                float4 out;
                if (s.bestSlot >= 0) {
                    const float* tb = reinterpret_cast<const float*>(tris + s.bestSlot);
                    const float4 A = ldg4(tb), B = ldg4(tb + 4), C = ldg4(tb + 8);
                    out.x = (float)RefineT(s.p.o, s.d, A, B, C);
                    out.y = A.w;  // input triangle index (bit pattern)
                    out.z = s.ba;
                    out.w = s.bb;
                } else {
                    out = make_float4(-1.0f, __int_as_float(-1), 0.0f, 0.0f);
                }
                *reinterpret_cast<float4*>(hits + ray) = out;
            }
            ray = -1;
        }
    }
}

namespace {

// Node visits per lane between ray refills of the eight-wide kernel.
constexpr int kW8Budget = 16;

template <bool ANY>
__global__ void __launch_bounds__(kTraceBlock, 8)
KTraceW8(const WNode8* __restrict__ nodes, const GpuTri* __restrict__ tris, const rtb200_ray* __restrict__ rays,
         long long n, rtb200_hit* __restrict__ hits, uint8_t* __restrict__ occ, unsigned long long* counter,
         unsigned* err)
{
    __shared__ uint2 sstack[kW8Stack * kTraceBlock];
    uint2* stk = sstack + threadIdx.x;
    WarpFeed feed{0ull, 0ull, false};
    W8State s;
    long long ray = -1;
    for (;;) {
        const long long got = FeedTake(feed, ray < 0, (unsigned long long)n, counter);
        if (got >= 0) {
            ray = got;
            StartRayW8(s, LoadRay(rays, ray));
        }
        if (__all_sync(kFull, ray < 0)) break;
        if (ray >= 0 && TraceW8<ANY>(s, nodes, tris, stk, err, kW8Budget)) {
            if (ANY) {
                occ[ray] = s.bestSlot >= 0 ? 1 : 0;
            } else {
                float4 out;
                if (s.bestSlot >= 0) {
                    const float* tb = reinterpret_cast<const float*>(tris + s.bestSlot);
                    const float4 A = ldg4(tb), B = ldg4(tb + 4), C = ldg4(tb + 8);
                    out.x = (float)RefineT(s.p.o, s.d, A, B, C);
                    out.y = A.w;
                    out.z = s.ba;
                    out.w = s.bb;
                } else {
                    out = make_float4(-1.0f, __int_as_float(-1), 0.0f, 0.0f);
                }
                *reinterpret_cast<float4*>(hits + ray) = out;
            }
            ray = -1;
        }
    }
}

template <class K>
int GridFor(K kernel, int num_sms)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTraceBlock, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * num_sms;
}

// One launch over `n` rays with the work counter and error word given.  The
// grid is the kernel's occupancy times the SM count, cached per instantiation
// and device (devices of one process may differ).
constexpr int kGridDevices = 64;

template <class NodeT, bool ANY, bool SPILL>
void Launch(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n, rtb200_hit* hits, uint8_t* occ,
            unsigned long long* counter, unsigned* err, cudaStream_t stream)
{
    static std::atomic<int> grids[kGridDevices];
    const int dev = s->ctx->device;
    int grid = (dev >= 0 && dev < kGridDevices) ? grids[dev].load(std::memory_order_relaxed) : 0;
    if (!grid) {
        grid = GridFor(KTrace<NodeT, ANY, SPILL>, s->ctx->num_sms);
        if (dev >= 0 && dev < kGridDevices) grids[dev].store(grid, std::memory_order_relaxed);
    }
    KTrace<NodeT, ANY, SPILL><<<grid, kTraceBlock, 0, stream>>>((const NodeT*)s->d_nodes, s->d_tris, d_rays, n,
                                                                (int)s->tri_material.size(), hits, occ, counter, err);
}

template <bool ANY>
cudaError_t Dispatch(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n, rtb200_hit* hits, uint8_t* occ,
                     unsigned long long* counter, unsigned* err, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const bool spill = s->stack_bound > kTraceStack;
    if (s->layout == RTB200_BVH_W8) {
        static std::atomic<int> grids[kGridDevices];
        const int dev = s->ctx->device;
        int grid = (dev >= 0 && dev < kGridDevices) ? grids[dev].load(std::memory_order_relaxed) : 0;
        if (!grid) {
            grid = GridFor(KTraceW8<ANY>, s->ctx->num_sms);
            if (dev >= 0 && dev < kGridDevices) grids[dev].store(grid, std::memory_order_relaxed);
        }
        KTraceW8<ANY><<<grid, kTraceBlock, 0, stream>>>((const WNode8*)s->d_nodes, s->d_tris, d_rays, n, hits, occ,
                                                        counter, err);
    } else if (s->layout == RTB200_BVH_Q8) {
        if (spill) Launch<QNode4, ANY, true>(s, d_rays, n, hits, occ, counter, err, stream);
        else Launch<QNode4, ANY, false>(s, d_rays, n, hits, occ, counter, err, stream);
    } else if (s->layout == RTB200_BVH_F16) {
        if (spill) Launch<HNode4, ANY, true>(s, d_rays, n, hits, occ, counter, err, stream);
        else Launch<HNode4, ANY, false>(s, d_rays, n, hits, occ, counter, err, stream);
    } else {
        if (spill) Launch<GpuNode4, ANY, true>(s, d_rays, n, hits, occ, counter, err, stream);
        else Launch<GpuNode4, ANY, false>(s, d_rays, n, hits, occ, counter, err, stream);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t LaunchCastClosest(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                              rtb200_hit* d_hits, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const cudaError_t e = cudaMemsetAsync(s->d_counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    return Dispatch<false>(s, d_rays, n, d_hits, nullptr, s->d_counter, s->d_err, stream);
}

cudaError_t LaunchCastClosestScratch(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                                     rtb200_hit* d_hits, unsigned long long* counter, unsigned* err,
                                     cudaStream_t stream)
{
    return Dispatch<false>(s, d_rays, n, d_hits, nullptr, counter, err, stream);
}

cudaError_t LaunchCastAnyScratch(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n, uint8_t* d_occ,
                                 unsigned long long* counter, unsigned* err, cudaStream_t stream)
{
    return Dispatch<true>(s, d_rays, n, nullptr, d_occ, counter, err, stream);
}

cudaError_t LaunchCastAny(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                          uint8_t* d_occ, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const cudaError_t e = cudaMemsetAsync(s->d_counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    return Dispatch<true>(s, d_rays, n, nullptr, d_occ, s->d_counter, s->d_err, stream);
}

}  // namespace rtb200
