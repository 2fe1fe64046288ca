// pathtrace.cu -- wavefront hero-wavelength spectral path tracer for sm_100a.
//
// Restates, as a wavefront, the reference's HWSS path loop
// (src/Library/Shaders/PathTracingIntegrator.cpp:3939-4821 IntegrateFromHitHWSS,
// :4855-5126 IntegrateRayHWSS) driven per pixel sample by
// PathTracingSpectralRasterizer::IntegratePixelSpectral
// (src/Library/Rendering/PathTracingSpectralRasterizer.cpp:121-198).
//
// A fixed pool of path slots lives in HBM as SoA.  One iteration is seven
// launches over device-side queues (no host round trip):
//   KAssign  split the free slots among the jobs that have samples left
//   KRegen   splat finished paths into the film, start new camera samples
//   KExtend  closest hit for every active path (warp while-while traversal)
//   KClassify sort the active paths by the material they hit
//   KShade   emission + MIS, next-event estimation to area lights and the
//            sky (shadow-ray queue), hero-wavelength BSDF sampling with
//            companion-wavelength weights, Russian roulette
//   KConnect any hit for the shadow-ray queue; unoccluded contributions are
//            added to the path's per-wavelength radiance
//   KSwap    rotate queue counters
// Appends to queues are warp-aggregated (one atomic per warp).
#include <cfloat>

#include "bsdf.cuh"
#include "core.h"
#include "env_map.h"
#include "pathtrace.h"
#include "pt_device.cuh"
#include "raycast.cuh"

namespace rtb200 {

constexpr int kShadeBlock = 256;
// Leaves tested per lane per traversal round in KExtend / KConnect (measured
// best for the path tracer's mixed secondary and shadow rays).
constexpr int kPathLeaves = 1;
constexpr float kInv4Pi = 0.07957747154594767f;

// ---- light BVH -------------------------------------------------------------

// LightBVH::NodeImportance (Lights/LightBVH.cpp:169-217) for full-sphere
// cones: power / max(squared distance from p to the node's box, 1e-4).
__device__ __forceinline__ float LightImportance(const PtLightNode* __restrict__ nodes, int i, V3 p)
{
    const float4 a = __ldg(reinterpret_cast<const float4*>(nodes + i));       // lo xyz, hi x
    const float4 b = __ldg(reinterpret_cast<const float4*>(nodes + i) + 1);   // hi yz, power, right
    if (!(b.z > 0.0f)) return 0.0f;
    const float lo[3] = {a.x, a.y, a.z}, hi[3] = {a.w, b.x, b.y}, q[3] = {p.x, p.y, p.z};
    float d2 = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float d = q[k] < lo[k] ? lo[k] - q[k] : (q[k] > hi[k] ? q[k] - hi[k] : 0.0f);
        d2 += d * d;
    }
    return b.z / fmaxf(d2, 1e-4f);
}

// LightBVH::Sample (LightBVH.cpp:423-482): from the root, pick a child in
// proportion to its importance, reusing the rescaled random number; returns
// the luminary and its selection probability (0: nothing to pick).
__device__ int SampleLightBvh(const PtLightNode* __restrict__ nodes, V3 p, float xi, float& pdf)
{
    pdf = 1.0f;
    int i = 0;
    for (int guard = 0; guard < 64; ++guard) {
        const int4 c = __ldg(reinterpret_cast<const int4*>(nodes + i) + 2);   // light, count, start, pad
        if (c.y <= 1) return c.x;
        const int right = __float_as_int(__ldg(reinterpret_cast<const float4*>(nodes + i) + 1).w);
        const float il = LightImportance(nodes, i + 1, p), ir = LightImportance(nodes, right, p);
        const float total = il + ir;
        if (!(total > 0.0f)) { pdf = 0.0f; return -1; }
        const float pl = il / total;
        if (xi < pl) {
            pdf *= pl;
            xi = xi / pl;
            i = i + 1;
        } else {
            pdf *= 1.0f - pl;
            xi = (xi - pl) / (1.0f - pl);
            i = right;
        }
    }
    pdf = 0.0f;
    return -1;
}

// LightBVH::Pdf (LightBVH.cpp:484-531): the probability that SampleLightBvh
// picks the luminary at leaf position `pos` from p.
__device__ float LightBvhPdf(const PtLightNode* __restrict__ nodes, int pos, V3 p)
{
    float pdf = 1.0f;
    int i = 0;
    for (int guard = 0; guard < 64; ++guard) {
        const int4 c = __ldg(reinterpret_cast<const int4*>(nodes + i) + 2);
        if (c.y <= 1) return pdf;
        const int right = __float_as_int(__ldg(reinterpret_cast<const float4*>(nodes + i) + 1).w);
        const float il = LightImportance(nodes, i + 1, p), ir = LightImportance(nodes, right, p);
        const float total = il + ir;
        if (!(total > 0.0f)) return 0.0f;
        const float pl = il / total;
        const int4 lc = __ldg(reinterpret_cast<const int4*>(nodes + i + 1) + 2);
        if (pos >= lc.z && pos < lc.z + lc.y) {
            pdf *= pl;
            i = i + 1;
        } else {
            pdf *= 1.0f - pl;
            i = right;
        }
    }
    return 0.0f;
}

// ---- image environment (env_map.h), out of line: rarely taken, and inlined
// it would add to the shading kernels' register pressure ----------------------

__device__ __noinline__ EnvSpec EnvLookupAt(const PtEnvMap* E, V3 d) { return EnvLookup(*E, d.x, d.y, d.z); }
__device__ __noinline__ float EnvPdfAt(const PtEnvMap* E, V3 d) { return EnvPdf(*E, d.x, d.y, d.z); }
__device__ __noinline__ float EnvSampleAt(const PtEnvMap* E, float u1, float u2, V3& d)
{
    return EnvSample(*E, u1, u2, d.x, d.y, d.z);
}

// ---- film ------------------------------------------------------------------

// XYZ of one finished sample: sum over active wavelengths of
// XYZ(lambda_i) * L_i, scaled by (lmax - lmin) / k_y / active
// (PathTracingSpectralRasterizer.cpp:141-198); a pixel sample of several
// spectral samples is their mean (1 / nSpectralSamples on the mean films; the
// filtered film's weights normalise it by themselves).
__device__ __forceinline__ void Splat(const PtPaths& P, const PtJobDev& J, int slot, uint4 m)
{
    const PtSettings& S = J.set;
    const float4 L = P.L[slot];
    const float hero = P.aux[slot].x;
    float lam[4];
    Wavelengths(hero, S.lmin, S.lmax, lam);
    const unsigned term = (m.z >> kTermShift) & 0xfu;
    float X = 0, Y = 0, Z = 0;
    int active = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float x, y, z;
        if (!(term & (1u << i)) && Cmf(lam[i], x, y, z)) {
            const float l = Get(L, i);
            X += x * l; Y += y * l; Z += z * l;
            ++active;
        }
    }
    if (active == 0) return;
    const float s = S.ynorm / (float)active * (S.filter == kFilterSplat ? 1.0f : S.inv_spectral);
    if (J.lum && Y != 0.0f) {
        // Adaptive sampling: the pixel's luminance sums for its convergence test.
        const double y = (double)(Y * s);
        atomicAdd(J.lum + 2 * (size_t)m.x, y);
        atomicAdd(J.lum + 2 * (size_t)m.x + 1, y * y);
    }
    if (S.filter != kFilterSplat) {
        float* px = J.film + 3 * (size_t)m.x;
        if (X != 0.0f) atomicAdd(px + 0, X * s);
        if (Y != 0.0f) atomicAdd(px + 1, Y * s);
        if (Z != 0.0f) atomicAdd(px + 2, Z * s);
        return;
    }
    // FilteredFilm::Splat (Rendering/FilteredFilm.cpp:42-98): the sample's
    // screen position (the camera's, see KRegen: uniform in its pixel, pixel
    // centres on integer coordinates) adds w XYZ and w to every pixel within the Gaussian's
    // support, w = exp(-r^2 / 2 sigma^2) / (2 pi sigma^2)
    // (GaussianPixelFilter.h:67-78).
    const int W = J.cam.width, H = J.cam.height;
    const int px = (int)(m.x % (uint32_t)W), py = (int)(m.x / (uint32_t)W);
    // The camera's jitter numbers again (hash key or Sobol seed in m.w, sample in m.y).
    const bool sobol = S.sampler != kSamplerHash, shuf = S.sampler == kSamplerSobolShuffled;
    const float ox = sobol ? SobolSample(m.y, 0, m.w, shuf) : Rand(m.w, 0);
    const float oy = sobol ? SobolSample(m.y, 1, m.w, shuf) : Rand(m.w, 1);
    const float sx = (float)px + ox - 0.5f, sy = (float)py + 0.5f - oy;
    const float hw = S.filt_half;
    const int x0 = max(0, (int)floorf(sx - hw)), x1 = min(W - 1, (int)floorf(sx + hw));
    const int y0 = max(0, (int)floorf(sy - hw)), y1 = min(H - 1, (int)floorf(sy + hw));
    X *= s; Y *= s; Z *= s;
    for (int qy = y0; qy <= y1; ++qy) {
        const float dy = sy - (float)qy;
        if (fabsf(dy) > hw) continue;
        for (int qx = x0; qx <= x1; ++qx) {
            const float dx = sx - (float)qx;
            if (fabsf(dx) > hw) continue;
            const float w = S.filt_norm * expf(-(dx * dx + dy * dy) * S.filt_inv2s2);
            float* f = J.film + 4 * ((size_t)qy * W + qx);
            if (X != 0.0f) atomicAdd(f + 0, X * w);
            if (Y != 0.0f) atomicAdd(f + 1, Y * w);
            if (Z != 0.0f) atomicAdd(f + 2, Z * w);
            atomicAdd(f + 3, w);
        }
    }
}

// ---- kernels ---------------------------------------------------------------

// Inclusive prefix sum over a block of up to 1024 threads.
__device__ __forceinline__ int BlockScan(int v, int* warp_sums)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) warp_sums[w] = v;
    __syncthreads();
    if (w == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(kFull, s, o);
            if (lane >= o) s += u;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    const int r = v + (w > 0 ? warp_sums[w - 1] : 0);
    __syncthreads();
    return r;
}

// Split this iteration's free slots among the jobs that still have camera
// samples (one block, one thread per job).  Every such job first gets a
// quarter of an equal share (capped by what it has left), so none starves;
// the rest goes to jobs in order of fewest samples left (shortest remaining
// first: in a serving mix the first progressive levels of new requests finish
// before long high-spp levels).  Each job's range of free-queue entries and
// first sample index go to Q.assign and its issued counter advances by its
// share.  Block prefix sums replace per-warp atomics on one counter per job.
// Images do not depend on this schedule: a sample's random numbers depend
// only on its job, pixel and sample index.
__global__ void __launch_bounds__(kPtMaxJobs)
KAssign(const PtJobDev* __restrict__ jobs, const int* __restrict__ ids, PtQueues Q, int iter)
{
    const int njobs = Q.cnt[kCntJobs];
    __shared__ int sums[32];
    __shared__ unsigned long long s_left[kPtMaxJobs];   // samples left per job (for the order)
    __shared__ int s_sorted[kPtMaxJobs];
    __shared__ int s_live, s_first;
    const int t = threadIdx.x;
    const int n = Q.cnt[kCntFree];
    int jid = -1, rem = 0;
    unsigned long long issued = 0, left_all = 0;
    if (t < njobs) {
        jid = ids[(t + iter) % njobs];
        const PtJobDev& J = jobs[jid];
        issued = *J.sample_ctr;
        if (issued < J.total) {
            left_all = J.total - issued;
            rem = (int)min(left_all, (unsigned long long)n);
        }
    }
    const int live = BlockScan(rem > 0 ? 1 : 0, sums);
    if (t == blockDim.x - 1) s_live = live;
    __syncthreads();
    const int share = s_live > 0 ? n / s_live / 4 : 0;
    const int first = min(rem, share);
    const int firstIncl = BlockScan(first, sums);
    if (t == blockDim.x - 1) s_first = firstIncl;
    s_left[t] = left_all;
    __syncthreads();
    const int left = n - s_first;
    const int more = rem - first;
    // Rank by samples left (ties by position), then a prefix sum in that order.
    int rank = 0;
    if (t < njobs)
        for (int k = 0; k < njobs; ++k) rank += (s_left[k] < left_all) || (s_left[k] == left_all && k < t);
    if (t < njobs) s_sorted[rank] = more;
    __syncthreads();
    const int v = t < njobs ? s_sorted[t] : 0;
    const int inclSorted = BlockScan(v, sums);
    s_sorted[t] = inclSorted - v;   // exclusive prefix in rank order
    __syncthreads();
    const int extra = t < njobs ? max(0, min(more, left - s_sorted[rank])) : 0;
    const int take = first + extra;
    const int takeIncl = BlockScan(take, sums);
    if (t < njobs) {
        PtAssign a;
        a.base = issued;
        a.off = takeIncl - take;
        a.jid = jid;
        Q.assign[t] = a;
        if (take > 0) *jobs[jid].sample_ctr = issued + (unsigned long long)take;
    }
    if (t == blockDim.x - 1) Q.cnt[kCntAssigned] = takeIncl;
}

__global__ void __launch_bounds__(kShadeBlock)
KRegen(const PtJobDev* __restrict__ jobs, PtPaths P, PtQueues Q, int assign)
{
    const int njobs = Q.cnt[kCntJobs];
    const int n = Q.cnt[kCntFree];
    const int nassigned = assign ? Q.cnt[kCntAssigned] : 0;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * 32; base < n; base += nwarps * 32) {
        const int i = base + lane;
        const bool valid = i < n;
        const int slot = valid ? Q.free_[i] : -1;
        int fin_job = -1;
        if (valid) {
            const uint4 m = P.meta[slot];
            if (m.z & kFlagFinishing) {
                fin_job = __float_as_int(P.aux[slot].z);
                Splat(P, jobs[fin_job], slot, m);
                P.meta[slot].z = m.z & ~kFlagFinishing;
            }
        }
        // Finished samples, one atomic per job present in the warp.
        const unsigned grp = __match_any_sync(kFull, fin_job);
        if (fin_job >= 0 && lane == __ffs(grp) - 1) atomicAdd(jobs[fin_job].done_ctr, (unsigned long long)__popc(grp));
        // New camera samples: free entry i < nassigned belongs to the job
        // whose assigned range holds it (KAssign).
        bool got = false;
        if (valid && i < nassigned) {
            int lo = 0, hi = njobs - 1;   // largest k with assign[k].off <= i
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (Q.assign[mid].off <= i) lo = mid; else hi = mid - 1;
            }
            const PtAssign a = Q.assign[lo];
            const int jid = a.jid;
            const PtJobDev& J = jobs[jid];
            const unsigned long long g = a.base + (unsigned long long)(i - a.off);
            {   // PinholeCamera::GenerateRay (Cameras/PinholeCamera.cpp:182-210)
                const uint32_t slot_px = (uint32_t)(g % (unsigned long long)J.npix);
                const uint32_t pixel = J.px_list ? __ldg(J.px_list + slot_px) : slot_px;
                const uint32_t sample = (uint32_t)(J.sample_begin + g / (unsigned long long)J.npix);
                const int px = (int)(pixel % (uint32_t)J.cam.width), py = (int)(pixel / (uint32_t)J.cam.width);
                const bool sobol = J.set.sampler != kSamplerHash, shuf = J.set.sampler == kSamplerSobolShuffled;
                // Hash key, or the pixel's Sobol seed (camera dimensions 0-2).
                const uint32_t key = sobol ? SobolPixelSeed((uint32_t)px, (uint32_t)py, J.set.seed)
                                           : PathKey(J.set.seed, pixel, sample);
                // Screen position in pixel units, pixel centres on integer
                // coordinates, rows counted downwards: the reference's
                // ptOnScreen = (x + u - 1/2, (height - y) + v - 1/2) for the
                // box filter and the filtered film
                // (PathTracingSpectralRasterizer.cpp:321-331, BoxPixelFilter.h:54-58),
                // or the pixel centre moved by the truncated Gaussian's
                // inverse CDF for a narrow Gaussian (GaussianPixelFilter.h:109-127).
                const float ox = sobol ? SobolSample(sample, 0, key, shuf) : Rand(key, 0);
                const float oy = sobol ? SobolSample(sample, 1, key, shuf) : Rand(key, 1);
                float fx, fy;
                if (J.set.filter == kFilterWarp) {
                    const float v = fmaxf(J.set.filt_trunc + (1.0f - J.set.filt_trunc) * ox, 1e-30f);
                    const float r = J.set.filt_sigma * sqrtf(-2.0f * logf(v));
                    float sn, cs;
                    sincospif(2.0f * oy, &sn, &cs);
                    fx = (float)px + r * cs;
                    fy = (float)py - r * sn;
                } else {
                    fx = (float)px + ox - 0.5f;
                    fy = (float)py + 0.5f - oy;
                }
                const float sx = 2.0f * fx / (float)J.cam.width - 1.0f;
                const float sy = 1.0f - 2.0f * fy / (float)J.cam.height;
                const V3 d = normalize(mk(J.cam.fwd[0] + sx * J.cam.right[0] + sy * J.cam.up[0],
                                          J.cam.fwd[1] + sx * J.cam.right[1] + sy * J.cam.up[1],
                                          J.cam.fwd[2] + sx * J.cam.right[2] + sy * J.cam.up[2]));
                // Wavelength: the hero of an equidistant bundle, or one
                // wavelength, binned as the reference's single-wavelength loop
                // bins it (lambda_begin + int(u * n) * step,
                // PathTracingSpectralRasterizer.cpp:180-183); the companions of a
                // single-wavelength path start terminated.
                const float uw = sobol ? SobolSample(sample, 2, key, shuf) : Rand(key, 2);
                const float hero = J.set.num_wl && J.set.single
                                       ? J.set.lmin + (float)min((int)(uw * (float)J.set.num_wl), J.set.num_wl - 1) *
                                                          J.set.wl_step
                                       : J.set.lmin + uw * (J.set.lmax - J.set.lmin);
                P.ray_o[slot] = make_float4(J.cam.pos[0], J.cam.pos[1], J.cam.pos[2], 0.0f);
                P.ray_d[slot] = make_float4(d.x, d.y, d.z, __int_as_float(0x7f800000));
                P.thr[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
                P.L[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                P.aux[slot] = make_float4(hero, 0.0f, __int_as_float(jid), 0.0f);
                P.meta[slot] = make_uint4(pixel, sample,
                                          kFlagConsiderEmission | (J.set.single ? (0xeu << kTermShift) : 0u), key);
                got = true;
            }
        }
        const int at = WarpAppend(&Q.cnt[kCntActive], got);
        if (got) Q.active[at] = slot;
        // Slots left without work stay queued for the next iteration, so
        // jobs submitted later find them.
        const bool idle = valid && !got;
        const int fi = WarpAppend(&Q.cnt[kCntFreeNext], idle);
        if (idle) Q.free_next[fi] = slot;
    }
}

// Closest hit for every active path.  Same while-while walk as KTrace; the
// hit stores the leaf-order triangle slot for shading.
// UNIFORM: every job shares the scene `us` (kernel argument, no per-path
// lookup of the job's scene).
template <class NodeT, bool SPILL, bool UNIFORM>
__global__ void __launch_bounds__(kTraceBlock, 8)
KExtend(const PtJobDev* __restrict__ jobs, PtPaths P, PtQueues Q, PtScene us)
{
    const NodeT* nodes = UNIFORM ? (const NodeT*)us.nodes : nullptr;
    const GpuTri* tris = UNIFORM ? us.tris : nullptr;
    int ntri = UNIFORM ? us.ntri : 0;
    __shared__ int sstack[kTraceStack * kTraceBlock];
    int spill[SPILL ? kTraceSpill : 1];
    const TraceStack stk{sstack + threadIdx.x, spill};
    const long long n = Q.cnt[kCntActive];
    WarpFeed feed{0ull, 0ull, false};
    TraceState s;
    long long qi = -1;
    int slot = -1;
    for (;;) {
        const long long got = FeedTake(feed, qi < 0, (unsigned long long)n, Q.trace_ctr);
        if (got >= 0) {
            qi = got;
            slot = Q.active[qi];
            if (!UNIFORM) {
                const PtScene& S = jobs[__float_as_int(P.aux[slot].z)].scene;
                nodes = (const NodeT*)S.nodes;
                tris = S.tris;
                ntri = S.ntri;
            }
            const float4 o = P.ray_o[slot], d = P.ray_d[slot];
            Ray r;
            r.o[0] = o.x; r.o[1] = o.y; r.o[2] = o.z; r.tmin = o.w;
            r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z; r.tmax = d.w;
            StartRay(s, r);
        }
        if (__all_sync(kFull, qi < 0)) break;
        if (qi >= 0 && TraceRound<NodeT, false, SPILL, kPathLeaves>(s, nodes, tris, ntri, stk, Q.err)) {
            P.hit[slot] = make_float4(s.best, __int_as_float(s.bestSlot), s.ba, s.bb);
            qi = -1;
        }
    }
}

// Any hit for the shadow-ray queue; unoccluded entries add their
// contribution to the path's radiance.
template <class NodeT, bool SPILL, bool UNIFORM>
__global__ void __launch_bounds__(kTraceBlock, 8)
KConnect(const PtJobDev* __restrict__ jobs, PtPaths P, PtQueues Q, PtScene us)
{
    const NodeT* nodes = UNIFORM ? (const NodeT*)us.nodes : nullptr;
    const GpuTri* tris = UNIFORM ? us.tris : nullptr;
    int ntri = UNIFORM ? us.ntri : 0;
    __shared__ int sstack[kTraceStack * kTraceBlock];
    int spill[SPILL ? kTraceSpill : 1];
    const TraceStack stk{sstack + threadIdx.x, spill};
    const long long n = Q.cnt[kCntShadow];
    WarpFeed feed{0ull, 0ull, false};
    TraceState s;
    long long qi = -1;
    for (;;) {
        const long long got = FeedTake(feed, qi < 0, (unsigned long long)n, Q.trace_ctr + 1);
        if (got >= 0) {
            qi = got;
            const ShadowEntry e = Q.shadow[qi];
            if (!UNIFORM) {
                const PtScene& S = jobs[__float_as_int(P.aux[__float_as_int(e.d.w)].z)].scene;
                nodes = (const NodeT*)S.nodes;
                tris = S.tris;
                ntri = S.ntri;
            }
            Ray r;
            r.o[0] = e.o.x; r.o[1] = e.o.y; r.o[2] = e.o.z; r.tmin = 0.0f;
            r.d[0] = e.d.x; r.d[1] = e.d.y; r.d[2] = e.d.z; r.tmax = e.o.w;
            StartRay(s, r);
        }
        if (__all_sync(kFull, qi < 0)) break;
        if (qi >= 0 && TraceRound<NodeT, true, SPILL, kPathLeaves>(s, nodes, tris, ntri, stk, Q.err)) {
            if (s.bestSlot < 0) {
                const ShadowEntry& e = Q.shadow[qi];
                const int slot = __float_as_int(e.d.w);
                float* l = reinterpret_cast<float*>(P.L + slot);
                if (e.c.x != 0.0f) atomicAdd(l + 0, e.c.x);
                if (e.c.y != 0.0f) atomicAdd(l + 1, e.c.y);
                if (e.c.z != 0.0f) atomicAdd(l + 2, e.c.z);
                if (e.c.w != 0.0f) atomicAdd(l + 3, e.c.w);
            }
            qi = -1;
        }
    }
}

__device__ __forceinline__ void PushShadow(const PtQueues& Q, V3 o, V3 d, float tmax, int slot, float4 c)
{
    const int at = WarpAppend(&Q.cnt[kCntShadow], true);
    ShadowEntry e;
    e.o = make_float4(o.x, o.y, o.z, tmax);
    e.d = make_float4(d.x, d.y, d.z, __int_as_float(slot));
    e.c = c;
    Q.shadow[at] = e;
}

// Wavelength-independent BSDF data of a next-event direction v seen from r:
// the GGX pair, or for Lambertian the same-side gate and pdf |nv|/pi
// (LambertianBRDF::valueNM + LambertianSPF::Pdf, ShouldReflect at
// LambertianBRDF.cpp:44-75).  The sampling pdf is wavelength-independent.
__device__ __forceinline__ GgxPair NeePair(int mtype, const GgxPoint& gp, V3 ns, V3 ng, V3 r, V3 v)
{
    if (mtype == kMatGGX) return GgxPairAt(gp, dot(r, ns) < 0.0f ? -ns : ns, ng, r, v);
    GgxPair q;
    const float nr = dot(ns, r), nv = dot(ns, v);
    const bool same = (nr >= kNearZero && nv >= kNearZero) || (nr <= -kNearZero && nv <= -kNearZero);
    q.ok = same && dot(v, ng) > 0.0f && dot(r, ng) > 0.0f;
    q.sf = q.rh = q.ms = 0.0f;
    q.pdf = q.ok ? fabsf(nv) * kInvPi : 0.0f;
    return q;
}

// Top of a path's index-of-refraction stack (entries from x upward, -1 past
// the top); the stack is read only when it holds a mesh.
__device__ __forceinline__ int MediaTop(int4 m)
{
    return m.w >= 0 ? m.w : (m.z >= 0 ? m.z : (m.y >= 0 ? m.y : m.x));
}

// The index a stack entry stands for: its dielectric's at the hero
// wavelength, as IORStack::push records it (DielectricSPF.cpp:198-207).
__device__ __noinline__ float MeshIor(const PtScene& S, int mesh, float lam)
{
    const PtMaterial M = S.mats[__ldg(S.mesh_mat + mesh)];
    return M.eta >= 0 ? Spec(S.spectra, M.eta, lam) : M.ior;
}

// The BSDF value at one wavelength for a next-event pair.
// The shading point's spectra at its four wavelengths, looked up once: the
// Lambertian reflectance or the GGX specular colour, the conductor's optical
// constants and its Fresnel average for the medium around the hit.
struct PointSpectra {
    float4 refl, eta, k, favg;
};

__device__ __forceinline__ GgxParams GgxOf(const PtMaterial& M, const PointSpectra& ps, int j, float amb)
{
    return GgxFrom(M, Get(ps.refl, j), Get(ps.eta, j), Get(ps.k, j), Get(ps.favg, j), amb);
}

// The BSDF value at wavelength j for a next-event pair.
__device__ __forceinline__ float NeeValue(int mtype, const PtMaterial& M, const PointSpectra& ps, int j,
                                          const GgxPair& q, float eavg, float amb)
{
    if (!q.ok) return 0.0f;
    if (mtype == kMatGGX) return GgxValueAt(q, GgxOf(M, ps, j, amb), eavg);
    return Get(ps.refl, j) * kInvPi;
}

// Sort the active paths into shading classes (escaped or Lambertian, GGX,
// dielectric) so KShade's warps each run one material model.
__global__ void __launch_bounds__(kShadeBlock)
KClassify(const PtJobDev* __restrict__ jobs, PtPaths P, PtQueues Q)
{
    const int n = Q.cnt[kCntActive];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int i = base + threadIdx.x;
        int cls = -1, slot = -1;
        if (i < n) {
            slot = Q.active[i];
            const int hslot = __float_as_int(P.hit[slot].y);
            cls = 0;
            if (hslot >= 0) {
                const PtScene& S = jobs[__float_as_int(P.aux[slot].z)].scene;
                const int type = S.mats[S.attr[hslot].mat & kAttrMatMask].type;
                cls = type == kMatGGX ? 1 : (type == kMatDielectric ? 2 : 0);
            }
        }
#pragma unroll
        for (int c = 0; c < kShadeClasses; ++c) {
            const int at = WarpAppend(&Q.cnt[kCntClass + c], cls == c);
            if (cls == c) Q.shade[c * Q.capacity + at] = slot;
        }
    }
}

// CLS >= 0: every path to shade escaped or hit a material of shading class
// CLS (0 Lambertian, 1 GGX, 2 dielectric), so the other models' code is left
// out and the kernel needs fewer registers; the paths come from KClassify's
// queue of that class (from_class) or, for scenes of one class, straight from
// the active queue.  CLS = -1 shades any material from the active queue.
// ENV: compiled with the image-environment code (some job's scene has one).
template <int CLS, bool ENV>
__global__ void __launch_bounds__(kShadeBlock, CLS == 1 || CLS < 0 ? 2 : 3)
KShade(const PtJobDev* __restrict__ jobs, PtPaths P, PtQueues Q, int from_class)
{
    const int n = (CLS >= 0 && from_class) ? Q.cnt[kCntClass + (CLS < 0 ? 0 : CLS)] : Q.cnt[kCntActive];
    const int* __restrict__ src = (CLS >= 0 && from_class) ? Q.shade + (CLS < 0 ? 0 : CLS) * Q.capacity : Q.active;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = src[i];
        const float4 aux = P.aux[slot];
        const PtJobDev& J = jobs[__float_as_int(aux.z)];
        const PtScene& S = J.scene;
        const PtSettings& set = J.set;
        uint4 m = P.meta[slot];
        const float4 h = P.hit[slot];
        const float4 ro = P.ray_o[slot], rd = P.ray_d[slot];
        float4 thr = P.thr[slot];
        float4 L = P.L[slot];
        const int depth = (int)(m.z & kFlagDepthMask);
        // Random numbers: hash key or Sobol seed in meta.w, sample index in meta.y.
        VertexRng rng{m.w, m.y, depth, set.sampler, 0u};
        const float bsdfPdf = aux.y;
        unsigned term = (m.z >> kTermShift) & 0xfu;
        float lam[4];
        Wavelengths(aux.x, set.lmin, set.lmax, lam);
        const V3 d = xyz(rd);
        bool cont = false;
        const int hslot = __float_as_int(h.y);

        do {
            if (hslot < 0) {
                // Escaped: uniform sky (IntegrateRayHWSS :5076-5120 for camera
                // rays; :4235-4303 with MIS against sky NEE for continuations),
                // or the image environment, weighted against its
                // importance sampling by EnvironmentSampler::Pdf (:4255-4283).
                if (ENV && S.env_map && (depth > 0 || set.env_visible)) {
                    const EnvSpec es = EnvLookupAt(S.env_map, d);
                    float w = 1.0f;
                    if (bsdfPdf > 0.0f) {
                        const float ep = EnvPdfAt(S.env_map, d);
                        if (ep > 0.0f) w = PowerHeuristic(bsdfPdf, ep);
                    }
                    for (int k = 0; k < 4; ++k)
                        if (!(term & (1u << k))) Set(L, k, Get(L, k) + Get(thr, k) * EnvSpectrum(es, lam[k]) * w);
                } else if (set.env >= 0 && (depth > 0 || set.env_visible)) {
                    const float w = bsdfPdf > 0.0f ? PowerHeuristic(bsdfPdf, kInv4Pi) : 1.0f;
                    for (int k = 0; k < 4; ++k)
                        if (!(term & (1u << k)))
                            Set(L, k, Get(L, k) + Get(thr, k) * Spec(S.spectra, set.env, lam[k]) * w);
                }
                break;
            }
            // Runaway-throughput guard (IntegrateFromHitHWSS :4094-4110).
            {
                float mx = 0.0f;
                bool bad = false;
                for (int k = 0; k < 4; ++k) {
                    const float v = Get(thr, k);
                    if (!isfinite(v)) bad = true;
                    mx = fmaxf(mx, fabsf(v));
                }
                if (bad || mx > 1e6f) break;
            }
            const float t = h.x;
            const V3 p = xyz(ro) + d * t;
            const float* tb = reinterpret_cast<const float*>(S.tris + hslot);
            const float4 A = ldg4(tb), B = ldg4(tb + 4), C = ldg4(tb + 8);
            const V3 nface = normalize(cross(xyz(B) - xyz(A), xyz(C) - xyz(A)));
            const PtTriAttr at = S.attr[hslot];
            const int mi = at.mat & kAttrMatMask;
            // Shading normal: the vertex normals interpolated at the hit,
            // n0 + (n1 - n0) a + (n2 - n0) b normalised, else the face normal
            // (TriangleMeshGeometryIndexedSpecializations.h:194-199,
            // Object.cpp:543); the geometric normal is the face normal turned
            // to the shading normal's side.
            V3 ns0 = nface;
            if (at.mat & kAttrSmooth) {
                const uint4 q = __ldg(S.tri_normals + hslot);
                const V3 n0 = OctDecode(q.x), n1 = OctDecode(q.y), n2 = OctDecode(q.z);
                ns0 = normalize(n0 + (n1 - n0) * h.z + (n2 - n0) * h.w);
            }
            V3 ng = dot(nface, ns0) < 0.0f ? -nface : nface;
            V3 ns = ns0;
            // Double-sided meshes turn both towards the incoming ray
            // (TriangleMeshGeometryIndexed.cpp:170-188).
            if (at.mat & kAttrDoubleSided) {
                if (dot(ns, d) > 0.0f) ns = -ns;
                if (dot(ng, d) > 0.0f) ng = -ng;
            }
            const V3 gnv = dot(ng, d) < 0.0f ? ng : -ng;   // geometric normal facing the ray
            const PtMaterial M = S.mats[mi];
            const int mtype = CLS < 0 ? M.type : CLS;
            // The path's index-of-refraction stack (IORStack.h); its top is
            // the medium around the hit, the ambient index of a conductor
            // (PathTracingIntegrator.cpp:4315-4322).  Lambertian shading
            // needs neither.
            int4 med = make_int4(-1, -1, -1, -1);
            float amb = 1.0f;
            if (CLS != 0 && (m.z & kFlagInMedium)) {
                med = P.media[slot];
                amb = MeshIor(S, MediaTop(med), lam[0]);
            }
            bool media_changed = false;

            // PART 1: emission with MIS against light sampling (:4424-4518).
            if (M.emit >= 0 && (m.z & kFlagConsiderEmission) && dot(-d, ng) > 0.0f) {
                float w = 1.0f;
                if (bsdfPdf > 0.0f && at.light >= 0) {
                    const PtLight lg = S.lights[at.light];
                    const float cosL = fabsf(dot(d, ng));
                    // Selection probability from the previous vertex (the ray's origin).
                    const float psel = (set.light_bvh && S.light_nodes) ? LightBvhPdf(S.light_nodes, lg.bvh_pos, xyz(ro))
                                                                         : lg.pdf;
                    if (cosL > 0.0f && lg.area > 0.0f) w = PowerHeuristic(bsdfPdf, psel * (t * t) / (lg.area * cosL));
                }
                for (int k = 0; k < 4; ++k)
                    if (!(term & (1u << k))) Set(L, k, Get(L, k) + Get(thr, k) * Spec(S.spectra, M.emit, lam[k]) * w);
            }

            float4 kray = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            V3 nd;
            float npdf = 0.0f;       // continuation pdf for the next emission MIS (0 = delta)
            unsigned nflags = kFlagConsiderEmission;
            int btype = kBounceDiffuse;   // ScatteredRay type of the continuation

            if (mtype == kMatDielectric) {
                // Smooth dielectric: Fresnel choice between reflection and
                // refraction (DielectricSPF.cpp:120-300) at the hero's index.
                // With a constant index every wavelength follows the hero's
                // direction with the same weight, so the bundle continues
                // together; where a companion's index differs from the hero's
                // (by more than 1e-8, GetSpecularInfoNM), the companions end
                // and the hero goes on alone (TerminateSecondary,
                // PathTracingIntegrator.cpp:4658-4677).
                const float ior = M.eta >= 0 ? Spec(S.spectra, M.eta, lam[0]) : M.ior;
                if (M.eta >= 0 && (term & 0xeu) != 0xeu) {
                    #pragma unroll 1
                    for (int k = 1; k < 4; ++k) {
                        if (!(term & (1u << k)) && fabsf(Spec(S.spectra, M.eta, lam[k]) - ior) > 1e-8f) {
                            term |= 0xeu;
                            m.z |= 0xeu << kTermShift;
                            break;
                        }
                    }
                }
                // Inside or outside from the stack, not the facing
                // (DielectricSPF.cpp:406-418): inside, the ray leaves for the
                // medium under this mesh's entry (:177-183); outside, it comes
                // from the stack's top (:198-207).  w is ri.onb.w(), the
                // shading normal turned towards the ray on a double-sided mesh.
                const int mesh = at.light >= 0 ? S.lights[at.light].mesh : ~at.light;
                int e[kPtMediaDepth] = {med.x, med.y, med.z, med.w};
                int depthIn = 0, pos = -1;
                #pragma unroll
                for (int i = 0; i < kPtMediaDepth; ++i) {
                    if (e[i] >= 0) depthIn = i + 1;
                    if (e[i] == mesh) pos = i;
                }
                const bool fromInside = pos >= 0;
                float exitIor = 1.0f;
                if (fromInside) {
                    const int below = pos == depthIn - 1 ? (depthIn >= 2 ? e[depthIn - 2] : -1) : e[depthIn - 1];
                    if (below >= 0) exitIor = MeshIor(S, below, lam[0]);
                }
                const float n1 = fromInside ? ior : amb, n2 = fromInside ? exitIor : ior;
                const V3 w = ns;
                const V3 nEff = fromInside ? -w : w;
                const V3 geomN = dot(ng, nEff) >= 0.0f ? ng : -ng;
                // Snell's law with the normal turned against the ray
                // (Optics.cpp:84-98); Fresnel on absolute cosines (:101-159).
                const V3 nf = dot(w, d) > 0.0f ? -w : w;
                const float cosI = -dot(d, nf);
                const float eta = n1 / n2;
                const float s2t = eta * eta * fmaxf(0.0f, 1.0f - cosI * cosI);
                const bool snell = 1.0f - s2t >= kNearZero;
                float R = 1.0f;
                V3 tdir = mk(0.0f, 0.0f, 0.0f);
                if (snell) {
                    const float cosT = sqrtf(1.0f - s2t);
                    tdir = normalize(d * eta + nf * (eta * cosI - cosT));
                    R = DielectricR(cosI, cosT, n1, n2);
                }
                // ScatterNM's two numbers (DielectricSPF.cpp:421) tilt the
                // transmitted direction by a Phong lobe of the material's
                // exponent: acos(u^(1/(n+1))) off it, uniform in azimuth
                // (GenerateScatteredRay, :248-272; none at 0 or >= 1e6).
                const float u1 = rng.next(16), u2 = rng.next(17);
                bool refr = snell;
                if (refr && M.alpha > 0.0f && M.alpha < 1e6f) {
                    const float a = acosf(powf(u1, 1.0f / (M.alpha + 1.0f)));
                    if (a > 0.0f && a < 0.5f * kPi) {
                        V3 tx, ty;
                        Basis(tdir, tx, ty);
                        float sp, cp, sa, ca;
                        __sincosf(2.0f * kPi * u2, &sp, &cp);
                        sincosf(a, &sa, &ca);
                        tdir = normalize(tdir * ca + (tx * cp + ty * sp) * sa);
                    }
                }
                // The transmitted ray must cross to the far side of w's
                // crossing (:274-279); the reflected one must stay above the
                // geometric normal on that side, and under total internal
                // reflection mirrors about it instead (:221-243).
                if (refr && !(dot(tdir, nEff) < -kNearZero)) refr = false;
                V3 rdir = normalize(d - w * (2.0f * dot(d, w)));
                bool refl = true;
                if (!(dot(rdir, geomN) > 0.0f)) {
                    if (R >= 1.0f) rdir = normalize(d - geomN * (2.0f * dot(d, geomN)));
                    else refl = false;
                }
                // RandomlySelect over (transmitted 1 - R, reflected R)
                // (ScatteredRayContainer.cpp:43-70); a lobe the reference
                // drops ends the path here with the same expectation.  The
                // transmitted ray carries the stack with this mesh pushed or
                // removed (PathTracingIntegrator.cpp:4814-4816).
                if (rng.next(18) < 1.0f - R) {
                    if (!refr) break;
                    nd = tdir;
                    btype = kBounceTransmission;
                    if (fromInside) {
                        #pragma unroll
                        for (int i = 0; i < kPtMediaDepth - 1; ++i)
                            if (i >= pos) e[i] = e[i + 1];
                        e[kPtMediaDepth - 1] = -1;
                    } else {
                        if (depthIn == kPtMediaDepth) break;   // deeper than the stack kept per path
                        #pragma unroll
                        for (int i = 0; i < kPtMediaDepth; ++i)
                            if (i == depthIn) e[i] = mesh;
                    }
                    med = make_int4(e[0], e[1], e[2], e[3]);
                    media_changed = true;
                } else {
                    if (!refl) break;
                    nd = rdir;
                    btype = kBounceGlossy;
                }
                for (int k = 0; k < 4; ++k) Set(kray, k, (term & (1u << k)) ? 0.0f : 1.0f);
                nflags |= kFlagSpecular;
            } else {
                const V3 r = -d;
                GgxPoint gp{1.0f, 0.0f, 0.0f, 0.0f};
                PointSpectra ps;
                ps.refl = ps.eta = ps.k = ps.favg = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (mtype == kMatGGX) {
                    gp = GgxPointAt(M.alpha, fabsf(dot(r, ns)));
                    #pragma unroll 1
                    for (int k = 0; k < 4; ++k) {
                        const float e = M.eta >= 0 ? Spec(S.spectra, M.eta, lam[k]) : M.ior;
                        const float kk = M.kappa >= 0 ? Spec(S.spectra, M.kappa, lam[k]) : 0.0f;
                        Set(ps.refl, k, M.refl >= 0 ? Spec(S.spectra, M.refl, lam[k]) : 1.0f);
                        Set(ps.eta, k, e);
                        Set(ps.k, k, kk);
                        Set(ps.favg, k, GgxFavg(M, S.spectra, lam[k], amb, e, kk));
                    }
                } else {
                    #pragma unroll 1
                    for (int k = 0; k < 4; ++k) Set(ps.refl, k, Spec(S.spectra, M.refl, lam[k]));
                }
                // PART 2: next-event estimation (LightSampler::EvaluateDirectLightingNM,
                // LightSampler.cpp:1942-2361): one area-light sample and one sky
                // sample per wavelength (reference) or one shared sample.
                const int nsamp = set.nee_per_lambda ? 4 : 1;
                #pragma unroll 1
                for (int k = 0; k < nsamp; ++k) {
                    if (set.nee_per_lambda && (term & (1u << k))) continue;
                    if (set.n_lights > 0) {
                        const float ul = rng.next(4 * k + 0);
                        int li = 0;
                        float psel;
                        if (set.light_bvh && S.light_nodes) {
                            li = SampleLightBvh(S.light_nodes, p, ul, psel);
                        } else {
                            // Alias table (AliasTable::Sample): one number
                            // picks an entry and decides between it and its alias.
                            const float sc = ul * (float)set.n_lights;
                            const int idx = min((int)sc, set.n_lights - 1);
                            const PtLightAlias al = S.light_alias[idx];
                            li = (sc - (float)idx < al.prob) ? idx : al.alias;
                            psel = S.lights[li].pdf;
                        }
                        // No sample when nothing can be picked, nor from a luminary to itself.
                        if (li >= 0 && S.lights[li].kind == 1 && psel > 0.0f) {
                            // Point light (LightSampler.cpp:2097-2130): luminance of
                            // colour x power, cos / d^2, no MIS (a delta light).
                            const PtLight lg = S.lights[li];
                            V3 toL = mk(lg.pos[0], lg.pos[1], lg.pos[2]) - p;
                            const float dist = sqrtf(dot(toL, toL));
                            toL = toL * (1.0f / dist);
                            const float cosS = dot(toL, ns);
                            if (dist > 0.0f && cosS > 0.0f) {
                                float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                                bool any = false;
                                const GgxPair bq = NeePair(mtype, gp, ns, gnv, r, toL);
                                #pragma unroll 1
                                for (int j = 0; j < 4; ++j) {
                                    if (term & (1u << j)) continue;
                                    if (set.nee_per_lambda && j != k) continue;
                                    const float f = NeeValue(mtype, M, ps, j, bq, gp.eavg, amb);
                                    const float v = Get(thr, j) * lg.le * f * cosS / (dist * dist) / psel;
                                    Set(c, j, v);
                                    any |= v != 0.0f;
                                }
                                if (any) PushShadow(Q, OffsetRay(p, ng, toL), toL, dist - 0.001f, slot, c);
                            }
                        } else if (li >= 0 && li != at.light && psel > 0.0f) {
                            const PtLight lg = S.lights[li];
                            const float ux = rng.next(4 * k + 1);
                            const float uy = rng.next(4 * k + 2);
                            const float uz = rng.next(4 * k + 3);
                            // First triangle whose area CDF reaches uz: binary
                            // search (std::lower_bound over the areas CDF,
                            // TriangleMeshGeometryIndexed.cpp:207-217).
                            int tsel = lg.first, hi = lg.first + lg.count - 1;
                            while (tsel < hi) {
                                const int mid = (tsel + hi) >> 1;
                                if (__ldg(&S.light_tris[mid].cdf) >= uz) hi = mid;
                                else tsel = mid + 1;
                            }
                            const PtLightTri lt = S.light_tris[tsel];
                            // GeometricUtilities::PointOnTriangle (GeometricUtilities.cpp:543-569).
                            const float sa = sqrtf(1.0f - ux);
                            const float alpha = 1.0f - sa, beta = sa * uy;
                            const V3 e1 = mk(lt.e1[0], lt.e1[1], lt.e1[2]), e2 = mk(lt.e2[0], lt.e2[1], lt.e2[2]);
                            const V3 pl = mk(lt.v0[0], lt.v0[1], lt.v0[2]) + e1 * alpha + e2 * beta;
                            const V3 nl = normalize(cross(e1, e2));
                            V3 toL = pl - p;
                            const float dist = sqrtf(dot(toL, toL));
                            toL = toL * (1.0f / dist);
                            const float cosS = dot(toL, ns);
                            const float cosL = dot(-toL, nl);
                            if (cosL > 0.0f && cosS > 0.0f) {
                                const float geom = lg.area * cosL / (dist * dist);
                                const float plight = psel * (dist * dist) / (lg.area * cosL);
                                float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                                bool any = false;
                                const GgxPair bq = NeePair(mtype, gp, ns, gnv, r, toL);
                                const float pb = bq.pdf;
                                #pragma unroll 1
                                for (int j = 0; j < 4; ++j) {
                                    if (term & (1u << j)) continue;
                                    if (set.nee_per_lambda && j != k) continue;
                                    const float f = NeeValue(mtype, M, ps, j, bq, gp.eavg, amb);
                                    const float w = (pb > 0.0f ? PowerHeuristic(plight, pb) : 1.0f) / psel;
                                    const float v = Get(thr, j) * Spec(S.spectra, lg.emit, lam[j]) * cosS * geom * f * w;
                                    Set(c, j, v);
                                    any |= v != 0.0f;
                                }
                                if (any) PushShadow(Q, OffsetRay(p, ng, toL), toL, dist - 0.001f, slot, c);
                            }
                        } else if (!(li >= 0 && S.lights[li].kind == 1 && psel > 0.0f)) {
                            // Nothing to sample, or the luminary being shaded:
                            // the reference still draws the point's three
                            // numbers (LightSampler.cpp:2064-2096).
                            rng.skip(3);
                        }
                    }
                    if (set.env >= 0 || (ENV && S.env_map)) {
                        // Environment NEE (LightSampler.cpp:2271-2359): the
                        // image environment's importance table
                        // (EnvironmentSampler::Sample), or for a uniform sky
                        // uniform directions with pdf 1/(4 pi).
                        const float u1 = rng.next(20 + 2 * k);
                        const float u2 = rng.next(21 + 2 * k);
                        V3 dir;
                        float epdf;
                        EnvSpec es{0.0f, 0.0f, 0.0f, 0.0f};
                        if (ENV && S.env_map) {
                            epdf = EnvSampleAt(S.env_map, u1, u2, dir);
                            if (epdf > 0.0f) es = EnvLookupAt(S.env_map, dir);
                        } else {
                            const float z = 1.0f - 2.0f * u1;
                            const float rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
                            float sp, cp;
                            __sincosf(2.0f * kPi * u2, &sp, &cp);
                            dir = mk(rr * cp, rr * sp, z);
                            epdf = kInv4Pi;
                        }
                        const float cosE = dot(dir, ns);
                        if (cosE > 0.0f && epdf > 0.0f) {
                            float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                            bool any = false;
                            const GgxPair bq = NeePair(mtype, gp, ns, gnv, r, dir);
                            const float pb = bq.pdf;
                            #pragma unroll 1
                            for (int j = 0; j < 4; ++j) {
                                if (term & (1u << j)) continue;
                                if (set.nee_per_lambda && j != k) continue;
                                const float f = NeeValue(mtype, M, ps, j, bq, gp.eavg, amb);
                                const float w = pb > 0.0f ? PowerHeuristic(epdf, pb) : 1.0f;
                                const float le = (ENV && S.env_map) ? EnvSpectrum(es, lam[j])
                                                                    : Spec(S.spectra, set.env, lam[j]);
                                const float v = Get(thr, j) * le * f * cosE / epdf * w;
                                Set(c, j, v);
                                any |= v != 0.0f;
                            }
                            if (any) PushShadow(Q, OffsetRay(p, ng, dir), dir, __int_as_float(0x7f800000), slot, c);
                        }
                    }
                }

                // PART 3: hero-wavelength BSDF sample (:4597-4719).
                const V3 w = dot(d, ns) > kNearZero ? -ns : ns;   // viewer side
                const V3 gn = gnv;
                V3 tx, ty;
                Basis(w, tx, ty);
                // GGXSPF::ScatterNM draws the lobe choice before the
                // direction (GGXSPF.cpp:478-520); LambertianSPF the direction.
                const float ulobe = mtype == kMatGGX ? rng.next(18) : 0.0f;
                const float u1 = rng.next(16), u2 = rng.next(17);
                if (mtype == kMatGGX) {
                    const GgxParams g0 = GgxOf(M, ps, 0, amb);
                    const float cosR = dot(r, w);
                    const float ws = g0.spec;
                    const float wms = ws * (1.0f - gp.essR);
                    const float total = ws + wms;
                    if (!(total > 1e-10f)) break;
                    const float pSpec = ws / total, pMS = wms / total;
                    const float msz = gp.msz;
                    float khero = 0.0f;
                    if (ulobe < pSpec) {
                        btype = kBounceGlossy;
                        const V3 mh = VndfSample(r, tx, ty, w, g0.alpha, u1, u2);
                        const float rm = dot(r, mh);
                        if (!(rm > 0.0f)) break;
                        nd = normalize(mh * (2.0f * rm) - r);
                        const float cosO = dot(nd, w);
                        if (!(cosO > 0.0f && dot(nd, gn) > 0.0f)) break;
                        const float vpdf = VndfPdf(r, nd, w, g0.alpha);
                        if (!(vpdf > 1e-10f)) break;
                        npdf = (wms * MsPdf(cosO, g0.alpha, msz) + ws * vpdf) / total;
                        const float G2 = 1.0f / (1.0f + GgxLambda(g0.alpha, cosR) + GgxLambda(g0.alpha, cosO));
                        const float G1 = 1.0f / (1.0f + GgxLambda(g0.alpha, cosR));
                        khero = g0.spec * ConductorF(rm, amb, g0.eta, g0.k) * G2 / (G1 * pSpec);
                    } else {
                        // Multiple-scattering lobe: mu_o from (1 - E(mu_o)) mu_o,
                        // uniform azimuth (GGXSPF.cpp:604-675).
                        const float eavg = gp.eavg;
                        if (!(pMS > 1e-10f && 1.0f - eavg > 1e-10f)) break;
                        const float cost = MsSampleCos(g0.alpha, u1);
                        const float sint = sqrtf(fmaxf(0.0f, 1.0f - cost * cost));
                        float sp, cp;
                        __sincosf(2.0f * kPi * u2, &sp, &cp);
                        nd = normalize(tx * (cp * sint) + ty * (sp * sint) + w * cost);
                        const float cosO = dot(nd, w);
                        if (!(cosO > 0.0f && dot(nd, gn) > 0.0f)) break;
                        const float mpdf = MsPdf(cosO, g0.alpha, msz);
                        if (!(mpdf > 1e-14f)) break;
                        npdf = (wms * mpdf + ws * VndfPdf(r, nd, w, g0.alpha)) / total;
                        const float fms = Fms(g0.spec * g0.favg, eavg) * (1.0f - LookupEss(cosO, g0.alpha)) *
                                          (1.0f - gp.essR) / (kPi * (1.0f - eavg));
                        khero = fms * cosO / (mpdf * pMS);
                    }
                    if (!(npdf > 0.0f)) break;
                    Set(kray, 0, (term & 1u) ? 0.0f : khero);
                    const float cosV = fabsf(dot(nd, ns));
                    // Companions evaluate the BSDF in the hero's direction and
                    // divide by the hero's pdf (:4676-4714).
                    const GgxPair cq = GgxPairAt(gp, w, gnv, r, nd);
                    #pragma unroll 1
                    for (int k = 1; k < 4; ++k) {
                        if (term & (1u << k)) continue;
                        Set(kray, k, GgxValueAt(cq, GgxOf(M, ps, k, amb), gp.eavg) * cosV / npdf);
                    }
                } else {
                    // Lambertian: cosine-weighted direction, kray = rho(lambda),
                    // pdf = cos/pi (LambertianSPF.cpp:90-160).
                    const float phi = 2.0f * kPi * u1;
                    const float sint = sqrtf(u2), cost = sqrtf(1.0f - u2);
                    float sp, cp;
                    __sincosf(phi, &sp, &cp);
                    nd = normalize(tx * (cp * sint) + ty * (sp * sint) + w * cost);
                    npdf = fabsf(dot(nd, w)) * kInvPi;
                    // Geometric-horizon gate (LambertianSPF.cpp:141-151).
                    if (!(dot(nd, gn) > 0.0f)) break;
                    for (int k = 0; k < 4; ++k) Set(kray, k, (term & (1u << k)) ? 0.0f : Get(ps.refl, k));
                }
                // The integrator's choice among the scattered rays
                // (ScatteredRayContainer::RandomlySelect; one ray here).
                rng.skip(1);
            }
            // Russian roulette on the max over wavelengths (:4738-4769,
            // PathTransportUtilities.h:86-110).
            float prevMax = 0.0f, currMax = 0.0f;
            for (int k = 0; k < 4; ++k) {
                if (term & (1u << k)) continue;
                prevMax = fmaxf(prevMax, fabsf(Get(thr, k)));
                currMax = fmaxf(currMax, fabsf(Get(thr, k) * Get(kray, k)));
            }
            if (currMax <= kNearZero) break;
            if (depth >= set.rr_min_depth) {
                const float prob = fminf(1.0f, currMax / fmaxf(prevMax, set.rr_threshold));
                if (rng.next(19) >= prob) break;
                if (prob > 0.0f && prob < 1.0f) {
                    const float s = 1.0f / prob;
                    kray = make_float4(kray.x * s, kray.y * s, kray.z * s, kray.w * s);
                }
            }
            // Per-type bounce limits (PropagateBounceLimits,
            // PathTransportUtilities.h:170-221), checked after Russian roulette
            // as the reference does (:4770-4790).
            unsigned bounces = __float_as_uint(aux.w);
            {
                const unsigned c = ((bounces >> (8 * btype)) & 0xffu) + 1u;
                if ((int)c > set.max_bounce[btype]) break;
                bounces = (bounces & ~(0xffu << (8 * btype))) | (c << (8 * btype));
            }
            if (depth + 1 >= set.max_depth) break;
            thr = make_float4(thr.x * kray.x, thr.y * kray.y, thr.z * kray.z, thr.w * kray.w);
            const V3 no = OffsetRay(p, nface, nd);
            P.ray_o[slot] = make_float4(no.x, no.y, no.z, 0.0f);
            P.ray_d[slot] = make_float4(nd.x, nd.y, nd.z, __int_as_float(0x7f800000));
            P.thr[slot] = thr;
            P.aux[slot] = make_float4(aux.x, npdf, aux.z, __uint_as_float(bounces));
            m.z = (m.z & ~(kFlagDepthMask | kFlagSpecular)) | (unsigned)(depth + 1) | nflags;
            if (media_changed) {
                P.media[slot] = med;
                m.z = med.x >= 0 ? (m.z | kFlagInMedium) : (m.z & ~kFlagInMedium);
            }
            P.meta[slot].z = m.z;
            cont = true;
        } while (false);

        P.L[slot] = L;
        if (!cont) P.meta[slot].z = m.z | kFlagFinishing;
        const int an = WarpAppend(&Q.cnt[kCntActiveNext], cont);
        if (cont) Q.active_next[an] = slot;
        const int fn = WarpAppend(&Q.cnt[kCntFreeNext], !cont);
        if (!cont) Q.free_next[fn] = slot;
    }
}

__global__ void KSwap(int* cnt)
{
    for (int c = 0; c < kShadeClasses; ++c) cnt[kCntClass + c] = 0;
    cnt[kCntSegments] += cnt[kCntActive];
    cnt[kCntShadowRays] += cnt[kCntShadow];
    cnt[kCntActive] = cnt[kCntActiveNext];
    cnt[kCntActiveNext] = 0;
    cnt[kCntFree] = cnt[kCntFreeNext];
    cnt[kCntFreeNext] = 0;
    cnt[kCntShadow] = 0;
}

// Kahan-compensated fold of this call's film into the running sums.
__global__ void KFold(float* pass, float* sum, float* comp, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float y = pass[i] - comp[i];
        const float s = sum[i];
        const float t = s + y;
        comp[i] = (t - s) - y;
        sum[i] = t;
        pass[i] = 0.0f;
    }
}

// Fold into the FP64 running sum used past 4096 spp; `first` moves the
// compensated FP32 sum over.
__global__ void KFoldWide(float* pass, float* sum, float* comp, double* wide, int n, int first)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double w = first ? (double)sum[i] - (double)comp[i] : wide[i];
        wide[i] = w + (double)pass[i];
        pass[i] = 0.0f;
        if (first) sum[i] = comp[i] = 0.0f;
    }
}

__device__ __forceinline__ double FilmValue(const float* __restrict__ sum, const float* __restrict__ comp,
                                            const double* __restrict__ wide, int k)
{
    return wide ? wide[k] : (double)sum[k] - (double)comp[k];
}

// relMSE of the resolved film (FP32 compensated or FP64 sums; 3 channels:
// sum / spp, 4 channels: weighted sum / weight, 0 where the weight is at most
// 1e-10) against `ref` (XYZ per pixel): sum over pixels and channels of
// (x - r)^2 / (r^2 + 1e-2), in FP64.
__global__ void KRelMse(const float* __restrict__ sum, const float* __restrict__ comp, const double* __restrict__ wide,
                        const unsigned* __restrict__ counts, const float* __restrict__ ref, int npix, int channels,
                        double inv_spp, double* out)
{
    double acc = 0.0;
    const int n3 = 3 * npix;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        double x;
        if (channels == 3) {
            const unsigned c = counts ? counts[i / 3] : 1u;
            x = c ? FilmValue(sum, comp, wide, i) * (counts ? 1.0 / (double)c : inv_spp) : 0.0;
        } else {
            const int p = i / 3;
            const double w = FilmValue(sum, comp, wide, 4 * p + 3);
            x = fabs(w) > 1e-10 ? FilmValue(sum, comp, wide, 4 * p + i - 3 * p) / w : 0.0;
        }
        const double r = ref[i];
        acc += (x - r) * (x - r) / (r * r + 1e-2);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
    __shared__ double part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
        if (threadIdx.x == 0) atomicAdd(out, acc);
    }
}

// Adaptive sampling after a batch of `batch` samples for each listed pixel
// (PathTracingSpectralRasterizer.cpp:379-408 with the Welford mean / M2
// formed from the sums of Y and Y^2): adds the batch to the pixel's count,
// tests convergence once it has 32 samples, and appends pixels still below
// the maximum and not converged to `next`.
__global__ void KConverge(const unsigned* __restrict__ list, int n, const double* __restrict__ lum,
                          unsigned* __restrict__ count, int batch, int max_spp, double threshold,
                          unsigned* __restrict__ next, int* __restrict__ n_next)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned p = list[i];
        const unsigned c = count[p] + (unsigned)batch;
        count[p] = c;
        bool converged = false;
        if (c >= 32) {
            const double N = (double)c, s1 = lum[2 * (size_t)p], s2 = lum[2 * (size_t)p + 1];
            const double mean = s1 / N;
            const double m2 = fmax(s2 - s1 * mean, 0.0);
            const double se = sqrt(m2 / (N - 1.0) / N), ma = fabs(mean);
            if (ma > 1e-12) converged = se / ma < threshold * (1.0 - 4.0 / N);
            else converged = m2 < 1e-12 && c >= 64;
        }
        if (!converged && (int)c < max_spp) next[atomicAdd(n_next, 1)] = p;
    }
}

// ---- host launchers ----------------------------------------------------------

namespace {
template <class K>
int TraceGrid(K kernel, int sms)
{
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kTraceBlock, 0) != cudaSuccess || per < 1) per = 1;
    return per * sms;
}
}  // namespace

// Extension kernel (closest hits of the path queue) when `extend`, else the
// connection kernel (shadow rays); grids cached per instantiation.
template <class NodeT, bool SPILL, bool UNIFORM>
void LaunchTraceKernels(const PtLaunch& L, cudaStream_t st, bool extend)
{
    if (extend) {
        static int g = 0;
        if (!g) g = TraceGrid(KExtend<NodeT, SPILL, UNIFORM>, L.sms);
        KExtend<NodeT, SPILL, UNIFORM><<<g, kTraceBlock, 0, st>>>(L.jobs, L.paths, L.queues, L.scene);
    } else {
        static int g = 0;
        if (!g) g = TraceGrid(KConnect<NodeT, SPILL, UNIFORM>, L.sms);
        KConnect<NodeT, SPILL, UNIFORM><<<g, kTraceBlock, 0, st>>>(L.jobs, L.paths, L.queues, L.scene);
    }
}

template <class NodeT>
void LaunchTrace(const PtLaunch& L, cudaStream_t st, bool extend)
{
    if (L.spill) {
        if (L.uniform) LaunchTraceKernels<NodeT, true, true>(L, st, extend);
        else LaunchTraceKernels<NodeT, true, false>(L, st, extend);
    } else {
        if (L.uniform) LaunchTraceKernels<NodeT, false, true>(L, st, extend);
        else LaunchTraceKernels<NodeT, false, false>(L, st, extend);
    }
}

cudaError_t PtSetGgxTables(const float* ess, const float* eavg, const float* msz, const float* mscum,
                           const float* favg_x, const float* favg_w)
{
    cudaError_t e = cudaMemcpyToSymbol(g_ess, ess, sizeof(float) * kLut * kLut);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_eavg, eavg, sizeof(float) * kLut);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_msz, msz, sizeof(float) * kLut);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_mscum, mscum, sizeof(float) * kLut * (kLut + 2));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_favg_x, favg_x, sizeof(float) * kFavgNodes);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_favg_w, favg_w, sizeof(float) * kFavgNodes);
    return e;
}

template <int CLS>
void LaunchShade(const PtLaunch& L, int from_class, cudaStream_t st)
{
    const int grid = L.sms * 8;
    if (L.env_image) KShade<CLS, true><<<grid, kShadeBlock, 0, st>>>(L.jobs, L.paths, L.queues, from_class);
    else KShade<CLS, false><<<grid, kShadeBlock, 0, st>>>(L.jobs, L.paths, L.queues, from_class);
}

cudaError_t PtIteration(const PtLaunch& L, int iter, cudaStream_t st)
{
    const int shadeGrid = L.sms * 8;
    KAssign<<<1, kPtMaxJobs, 0, st>>>(L.jobs, L.ids, L.queues, iter);
    KRegen<<<shadeGrid, kShadeBlock, 0, st>>>(L.jobs, L.paths, L.queues, 1);
    cudaMemsetAsync(L.queues.trace_ctr, 0, 2 * sizeof(unsigned long long), st);
    if (L.layout == RTB200_BVH_Q8) LaunchTrace<QNode4>(L, st, true);
    else if (L.layout == RTB200_BVH_F16) LaunchTrace<HNode4>(L, st, true);
    else LaunchTrace<GpuNode4>(L, st, true);
    if (L.classify) {
        KClassify<<<shadeGrid, kShadeBlock, 0, st>>>(L.jobs, L.paths, L.queues);
        LaunchShade<0>(L, 1, st);
        LaunchShade<1>(L, 1, st);
        // Dielectrics shade neither escaped rays nor next events.
        KShade<2, false><<<shadeGrid, kShadeBlock, 0, st>>>(L.jobs, L.paths, L.queues, 1);
    } else if (L.shade_class == 0) {
        LaunchShade<0>(L, 0, st);
    } else if (L.shade_class == 1) {
        LaunchShade<1>(L, 0, st);
    } else if (L.shade_class == 2) {
        // A dielectric-only scene: this kernel also shades the escaped rays.
        LaunchShade<2>(L, 0, st);
    } else {
        LaunchShade<-1>(L, 0, st);
    }
    if (L.layout == RTB200_BVH_Q8) LaunchTrace<QNode4>(L, st, false);
    else if (L.layout == RTB200_BVH_F16) LaunchTrace<HNode4>(L, st, false);
    else LaunchTrace<GpuNode4>(L, st, false);
    KSwap<<<1, 1, 0, st>>>(L.queues.cnt);
    return cudaGetLastError();
}

cudaError_t PtDrain(const PtLaunch& L, cudaStream_t st)
{
    KRegen<<<L.sms * 8, kShadeBlock, 0, st>>>(L.jobs, L.paths, L.queues, 0);
    return cudaGetLastError();
}

cudaError_t PtFoldWide(float* pass, float* sum, float* comp, double* wide, int n, bool first, int sms,
                       cudaStream_t st)
{
    KFoldWide<<<sms * 4, 256, 0, st>>>(pass, sum, comp, wide, n, first ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t PtRelMse(const float* sum, const float* comp, const double* wide, const unsigned* counts,
                     const float* ref, int npix, int channels, double inv_spp, double* out, int sms, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
    if (e != cudaSuccess) return e;
    KRelMse<<<sms * 2, 256, 0, st>>>(sum, comp, wide, counts, ref, npix, channels, inv_spp, out);
    return cudaGetLastError();
}

cudaError_t PtConverge(const unsigned* list, int n, const double* lum, unsigned* count, int batch, int max_spp,
                       double threshold, unsigned* next, int* n_next, int sms, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(n_next, 0, sizeof(int), st);
    if (e != cudaSuccess || n == 0) return e;
    KConverge<<<std::min(sms * 8, (n + 255) / 256), 256, 0, st>>>(list, n, lum, count, batch, max_spp, threshold,
                                                                  next, n_next);
    return cudaGetLastError();
}

cudaError_t PtFold(float* pass, float* sum, float* comp, int n, int sms, cudaStream_t st)
{
    KFold<<<sms * 4, 256, 0, st>>>(pass, sum, comp, n);
    return cudaGetLastError();
}

}  // namespace rtb200
