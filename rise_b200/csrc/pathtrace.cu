// pathtrace.cu -- wavefront hero-wavelength spectral path tracer for sm_100a.
//
// Restates, as a wavefront, the reference's HWSS path loop
// (src/Library/Shaders/PathTracingIntegrator.cpp:3939-4821 IntegrateFromHitHWSS,
// :4855-5126 IntegrateRayHWSS) driven per pixel sample by
// PathTracingSpectralRasterizer::IntegratePixelSpectral
// (src/Library/Rendering/PathTracingSpectralRasterizer.cpp:121-198).
//
// A fixed pool of path slots lives in HBM as SoA.  One iteration is five
// launches over device-side queues (no host round trip):
//   KRegen   splat finished paths into the film, start new camera samples
//   KExtend  closest hit for every active path (warp while-while traversal)
//   KShade   emission + MIS, next-event estimation (shadow-ray queue),
//            hero-wavelength BSDF sampling, Russian roulette
//   KConnect any hit for the shadow-ray queue; unoccluded contributions are
//            added to the path's per-wavelength radiance
//   KSwap    rotate queue counters
// Appends to queues are warp-aggregated (one atomic per warp).
#include <cfloat>

#include "cie1931.h"
#include "core.h"
#include "pathtrace.h"
#include "raycast.cuh"

namespace rtb200 {

__constant__ float c_cie[3][RTB200_CIE_COUNT] = {{RTB200_CIE_XBAR}, {RTB200_CIE_YBAR}, {RTB200_CIE_ZBAR}};

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kNearZero = 1e-12f;   // NEARZERO, Utilities/Math3D/Constants.h:33
constexpr int kShadeBlock = 256;

// ---- random numbers --------------------------------------------------------
// Counter-based: every number is a hash of (seed, pixel, sample, dimension),
// so the oracle draws the identical sequence on the CPU.

__device__ __forceinline__ uint32_t Mix32(uint32_t x)
{
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ uint32_t PathKey(uint32_t seed, uint32_t pixel, uint32_t sample)
{
    return Mix32(Mix32(seed ^ 0x9e3779b9u ^ Mix32(pixel)) ^ sample);
}

__device__ __forceinline__ float Rand(uint32_t key, uint32_t dim)
{
    return (float)(Mix32(key ^ (dim * 0x9e3779b9u + 0x7f4a7c15u)) >> 8) * (1.0f / 16777216.0f);
}

// Dimension layout: camera jitter 0-1, hero wavelength 2; bounce `depth`
// uses 8 + 32*depth + j: NEE sample i at j = 4i..4i+3 (light, x, y, triangle),
// BSDF direction j = 16, 17, lobe selection 18, Russian roulette 19.
__device__ __forceinline__ uint32_t Dim(int depth, int j) { return 8u + 32u * (uint32_t)depth + (uint32_t)j; }

// ---- spectra ---------------------------------------------------------------

// Linear interpolation on the 5 nm grid (InterpSPDIndices,
// src/Library/Utilities/Color/ColorUtils.cpp:270-300); 0 outside 380..780 nm.
__device__ __forceinline__ float Spec(const float* spectra, int id, float nm)
{
    if (id < 0 || !(nm >= 380.0f) || nm > 780.0f) return 0.0f;
    const float x = (nm - 380.0f) * 0.2f;
    const int i = (int)floorf(x);
    const int j = i + 1 > 80 ? 80 : i + 1;
    const float w = x - (float)i;
    const float* s = spectra + id * RTB200_CIE_COUNT;
    return s[i] + w * (s[j] - s[i]);
}

// ColorUtils::XYZFromNM (ColorUtils.cpp:313-325).
__device__ __forceinline__ bool Cmf(float nm, float& X, float& Y, float& Z)
{
    if (!(nm >= 380.0f) || nm > 780.0f) return false;
    const float x = (nm - 380.0f) * 0.2f;
    const int i = (int)floorf(x);
    const int j = i + 1 > 80 ? 80 : i + 1;
    const float w = x - (float)i;
    X = c_cie[0][i] + w * (c_cie[0][j] - c_cie[0][i]);
    Y = c_cie[1][i] + w * (c_cie[1][j] - c_cie[1][i]);
    Z = c_cie[2][i] + w * (c_cie[2][j] - c_cie[2][i]);
    return true;
}

// SampledWavelengths::SampleEquidistant
// (src/Library/Utilities/Color/SampledWavelengths.h:79-106).
__device__ __forceinline__ void Wavelengths(float hero, float lmin, float lmax, float lam[4])
{
    const float range = lmax - lmin;
    const float delta = range * 0.25f;
    lam[0] = hero;
#pragma unroll
    for (int i = 1; i < 4; ++i) lam[i] = lmin + fmodf(hero - lmin + (float)i * delta, range);
}

__device__ __forceinline__ float Get(const float4& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }
__device__ __forceinline__ void Set(float4& v, int i, float x)
{
    if (i == 0) v.x = x; else if (i == 1) v.y = x; else if (i == 2) v.z = x; else v.w = x;
}

// ---- small vector helpers --------------------------------------------------

struct V3 { float x, y, z; };
__device__ __forceinline__ V3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ V3 normalize(V3 a) { return a * rsqrtf(fmaxf(dot(a, a), 1e-30f)); }
__device__ __forceinline__ V3 xyz(float4 v) { return {v.x, v.y, v.z}; }

// Orthonormal basis around unit n (Duff et al., JCGT 6(1), 2017).
__device__ __forceinline__ void Basis(V3 n, V3& t, V3& b)
{
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float c = n.x * n.y * a;
    t = mk(1.0f + sign * n.x * n.x * a, sign * c, -sign * n.x);
    b = mk(c, sign + n.y * n.y * a, -n.y);
}

// Ray origin pushed off the surface on the side of `dir` by a few float ulps
// (Waechter and Binder, "A Fast and Robust Method for Avoiding
// Self-Intersection", Ray Tracing Gems, 2019).  The reference advances the
// origin by 1e-8 along the ray in double precision
// (PathTracingIntegrator.cpp:4812); in FP32 that step is below one ulp.
__device__ __forceinline__ V3 OffsetRay(V3 p, V3 ng, V3 dir)
{
    const V3 n = dot(dir, ng) >= 0.0f ? ng : -ng;
    const float kOrigin = 1.0f / 32.0f, kFloat = 1.0f / 65536.0f, kInt = 256.0f;
    const int ox = (int)(kInt * n.x), oy = (int)(kInt * n.y), oz = (int)(kInt * n.z);
    const V3 pi = mk(__int_as_float(__float_as_int(p.x) + (p.x < 0 ? -ox : ox)),
                     __int_as_float(__float_as_int(p.y) + (p.y < 0 ? -oy : oy)),
                     __int_as_float(__float_as_int(p.z) + (p.z < 0 ? -oz : oz)));
    return mk(fabsf(p.x) < kOrigin ? p.x + kFloat * n.x : pi.x,
              fabsf(p.y) < kOrigin ? p.y + kFloat * n.y : pi.y,
              fabsf(p.z) < kOrigin ? p.z + kFloat * n.z : pi.z);
}

// PathTransportUtilities::PowerHeuristic (Utilities/PathTransportUtilities.h:251).
__device__ __forceinline__ float PowerHeuristic(float a, float b)
{
    const float a2 = a * a;
    return a2 / (a2 + b * b);
}

// ---- warp-aggregated queue append -----------------------------------------

__device__ __forceinline__ int WarpAppend(int* counter, bool pred)
{
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, pred);
    if (!m) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(act, base, leader);
    return pred ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

// ---- film ------------------------------------------------------------------

// XYZ of one finished sample: sum over active wavelengths of
// XYZ(lambda_i) * L_i, scaled by (lmax - lmin) / k_y / active
// (PathTracingSpectralRasterizer.cpp:141-174).
__device__ __forceinline__ void Splat(const PtPaths& P, const PtFilm& F, const PtSettings& S, int slot, uint4 m)
{
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
    const float s = S.ynorm / (float)active;
    float* px = F.pass + 3 * (size_t)m.x;
    if (X != 0.0f) atomicAdd(px + 0, X * s);
    if (Y != 0.0f) atomicAdd(px + 1, Y * s);
    if (Z != 0.0f) atomicAdd(px + 2, Z * s);
}

// ---- kernels ---------------------------------------------------------------

__global__ void __launch_bounds__(kShadeBlock)
KRegen(PtPaths P, PtQueues Q, PtFilm F, PtJobParams J)
{
    const int n = Q.cnt[kCntFree];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * 32; base < n; base += nwarps * 32) {
        const int i = base + lane;
        const bool valid = i < n;
        const int slot = valid ? Q.free_[i] : -1;
        if (valid) {
            const uint4 m = P.meta[slot];
            if (m.z & kFlagFinishing) {
                Splat(P, F, J.set, slot, m);
                P.meta[slot].z = m.z & ~kFlagFinishing;
            }
        }
        // Take new samples for the valid lanes (one atomic per warp).
        const unsigned want = __ballot_sync(kFull, valid);
        unsigned long long g0 = 0;
        if (lane == 0 && want) g0 = atomicAdd(Q.sample_ctr, (unsigned long long)__popc(want));
        g0 = __shfl_sync(kFull, g0, 0);
        const unsigned long long g = g0 + __popc(want & ((1u << lane) - 1u));
        const bool got = valid && g < J.total;
        if (got) {
            const uint32_t pixel = (uint32_t)(g % (unsigned long long)J.npix);
            const uint32_t sample = (uint32_t)(J.sample_begin + g / (unsigned long long)J.npix);
            const uint32_t key = PathKey(J.set.seed, pixel, sample);
            const int px = (int)(pixel % (uint32_t)J.cam.width), py = (int)(pixel / (uint32_t)J.cam.width);
            // Box pixel filter of width 1: uniform jitter inside the pixel.
            const float fx = (float)px + Rand(key, 0), fy = (float)py + Rand(key, 1);
            const float sx = 2.0f * fx / (float)J.cam.width - 1.0f;
            const float sy = 1.0f - 2.0f * fy / (float)J.cam.height;
            const V3 d = normalize(mk(J.cam.fwd[0] + sx * J.cam.right[0] + sy * J.cam.up[0],
                                      J.cam.fwd[1] + sx * J.cam.right[1] + sy * J.cam.up[1],
                                      J.cam.fwd[2] + sx * J.cam.right[2] + sy * J.cam.up[2]));
            const float hero = J.set.lmin + Rand(key, 2) * (J.set.lmax - J.set.lmin);
            P.ray_o[slot] = make_float4(J.cam.pos[0], J.cam.pos[1], J.cam.pos[2], 0.0f);
            P.ray_d[slot] = make_float4(d.x, d.y, d.z, __int_as_float(0x7f800000));
            P.thr[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
            P.L[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            P.aux[slot] = make_float4(hero, 0.0f, 0.0f, 0.0f);
            P.meta[slot] = make_uint4(pixel, sample, kFlagConsiderEmission, key);
        }
        const int at = WarpAppend(&Q.cnt[kCntActive], got);
        if (got) Q.active[at] = slot;
    }
}

// Closest hit for every active path.  Same while-while walk as KTrace; the
// hit stores the leaf-order triangle slot for shading.
template <class NodeT>
__global__ void __launch_bounds__(kTraceBlock, 8)
KExtend(const NodeT* __restrict__ nodes, PtScene S, PtPaths P, PtQueues Q)
{
    __shared__ int sstack[kTraceStack * kTraceBlock];
    int* stk = sstack + threadIdx.x;
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
            const float4 o = P.ray_o[slot], d = P.ray_d[slot];
            Ray r;
            r.o[0] = o.x; r.o[1] = o.y; r.o[2] = o.z; r.tmin = o.w;
            r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z; r.tmax = d.w;
            StartRay(s, r);
        }
        if (__all_sync(kFull, qi < 0)) break;
        if (qi >= 0 && TraceRound<NodeT, false>(s, nodes, S.tris, S.ntri, stk, Q.err)) {
            P.hit[slot] = make_float4(s.best, __int_as_float(s.bestSlot), s.ba, s.bb);
            qi = -1;
        }
    }
}

// Any hit for the shadow-ray queue; unoccluded entries add their
// contribution to the path's radiance.
template <class NodeT>
__global__ void __launch_bounds__(kTraceBlock, 8)
KConnect(const NodeT* __restrict__ nodes, PtScene S, PtPaths P, PtQueues Q)
{
    __shared__ int sstack[kTraceStack * kTraceBlock];
    int* stk = sstack + threadIdx.x;
    const long long n = Q.cnt[kCntShadow];
    WarpFeed feed{0ull, 0ull, false};
    TraceState s;
    long long qi = -1;
    for (;;) {
        const long long got = FeedTake(feed, qi < 0, (unsigned long long)n, Q.trace_ctr + 1);
        if (got >= 0) {
            qi = got;
            const ShadowEntry e = Q.shadow[qi];
            Ray r;
            r.o[0] = e.o.x; r.o[1] = e.o.y; r.o[2] = e.o.z; r.tmin = 0.0f;
            r.d[0] = e.d.x; r.d[1] = e.d.y; r.d[2] = e.d.z; r.tmax = e.o.w;
            StartRay(s, r);
        }
        if (__all_sync(kFull, qi < 0)) break;
        if (qi >= 0 && TraceRound<NodeT, true>(s, nodes, S.tris, S.ntri, stk, Q.err)) {
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

__device__ __forceinline__ void Finish(const PtPaths& P, const PtQueues& Q, int slot, uint4 m, bool& fin)
{
    P.meta[slot].z = m.z | kFlagFinishing;
    fin = true;
}

__global__ void __launch_bounds__(kShadeBlock)
KShade(PtScene S, PtPaths P, PtQueues Q, PtJobParams J)
{
    const int n = Q.cnt[kCntActive];
    const PtSettings& set = J.set;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = Q.active[i];
        uint4 m = P.meta[slot];
        const float4 h = P.hit[slot];
        const float4 ro = P.ray_o[slot], rd = P.ray_d[slot];
        float4 thr = P.thr[slot];
        float4 L = P.L[slot];
        const float4 aux = P.aux[slot];
        const int depth = (int)(m.z & kFlagDepthMask);
        const uint32_t key = m.w;
        const float bsdfPdf = aux.y;
        const unsigned term = (m.z >> kTermShift) & 0xfu;
        float lam[4];
        Wavelengths(aux.x, set.lmin, set.lmax, lam);
        const V3 d = xyz(rd);
        bool fin = false;
        bool cont = false;
        int nsh = 0;
        ShadowEntry sh[4];
        const int hslot = __float_as_int(h.y);

        do {
            if (hslot < 0) {
                // Escaped: uniform sky radiance (IntegrateRayHWSS :5076-5120 for the
                // camera ray, IntegrateFromHitHWSS :4235-4303 for continuations).
                if (set.env >= 0 && (depth > 0 || set.env_visible)) {
                    for (int k = 0; k < 4; ++k)
                        if (!(term & (1u << k))) Set(L, k, Get(L, k) + Get(thr, k) * Spec(S.spectra, set.env, lam[k]));
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
            V3 ng = normalize(cross(xyz(B) - xyz(A), xyz(C) - xyz(A)));
            const PtTriAttr at = S.attr[hslot];
            const int mi = at.mat & kAttrMatMask;
            // Double-sided meshes face the incoming ray
            // (TriangleMeshGeometryIndexed.cpp:170-188).
            if ((at.mat & kAttrDoubleSided) && dot(ng, d) > 0.0f) ng = -ng;
            const PtMaterial M = S.mats[mi];

            // PART 1: emission with MIS against light sampling (:4424-4518).
            if (M.emit >= 0 && (m.z & kFlagConsiderEmission) && dot(-d, ng) > 0.0f) {
                float w = 1.0f;
                if (bsdfPdf > 0.0f && at.light >= 0) {
                    const PtLight lg = S.lights[at.light];
                    const float cosL = fabsf(dot(d, ng));
                    if (cosL > 0.0f && lg.area > 0.0f) {
                        const float pnee = lg.pdf * (t * t) / (lg.area * cosL);
                        w = PowerHeuristic(bsdfPdf, pnee);
                    }
                }
                for (int k = 0; k < 4; ++k)
                    if (!(term & (1u << k))) Set(L, k, Get(L, k) + Get(thr, k) * Spec(S.spectra, M.emit, lam[k]) * w);
            }
            if (M.type != kMatLambertian) break;  // other models: see KShade extensions

            // Shading frame: flat triangles shade with the face normal; the
            // Lambertian SPF samples around the normal on the viewer's side
            // (LambertianSPF.cpp:90-160).
            const V3 ns = ng;
            const float viewCos = dot(-d, ns);

            // PART 2: next-event estimation to area lights
            // (LightSampler::EvaluateDirectLightingNM, LightSampler.cpp:2083-2271).
            if (set.n_lights > 0 && viewCos > kNearZero) {
                const int nsamp = set.nee_per_lambda ? 4 : 1;
                for (int k = 0; k < nsamp; ++k) {
                    if (set.nee_per_lambda && (term & (1u << k))) continue;
                    const float ul = Rand(key, Dim(depth, 4 * k + 0));
                    int li = 0;
                    {
                        float acc = 0.0f;
                        for (li = 0; li < set.n_lights - 1; ++li) {
                            acc += S.lights[li].pdf;
                            if (ul < acc) break;
                        }
                    }
                    if (li == at.light) continue;   // no self-illumination
                    const PtLight lg = S.lights[li];
                    const float ux = Rand(key, Dim(depth, 4 * k + 1));
                    const float uy = Rand(key, Dim(depth, 4 * k + 2));
                    const float uz = Rand(key, Dim(depth, 4 * k + 3));
                    // First triangle whose area CDF reaches uz (std::lower_bound).
                    int tsel = lg.first + lg.count - 1;
                    for (int q = lg.first; q < lg.first + lg.count; ++q)
                        if (S.light_tris[q].cdf >= uz) { tsel = q; break; }
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
                    if (cosL <= 0.0f || cosS <= 0.0f) continue;
                    const float geom = lg.area * cosL / (dist * dist);
                    // MIS: light pdf (solid angle) vs Lambertian pdf cos/pi.
                    const float plight = lg.pdf * (dist * dist) / (lg.area * cosL);
                    const float w = PowerHeuristic(plight, cosS * kInvPi) / lg.pdf;
                    float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    bool any = false;
                    for (int j = 0; j < 4; ++j) {
                        if (term & (1u << j)) continue;
                        if (set.nee_per_lambda && j != k) continue;
                        const float f = Spec(S.spectra, M.refl, lam[j]) * kInvPi;
                        const float v = Get(thr, j) * Spec(S.spectra, lg.emit, lam[j]) * cosS * geom * f * w;
                        Set(c, j, v);
                        any |= v != 0.0f;
                    }
                    if (!any) continue;
                    const V3 so = OffsetRay(p, ng, toL);
                    ShadowEntry& e = sh[nsh++];
                    e.o = make_float4(so.x, so.y, so.z, dist - 0.001f);
                    e.d = make_float4(toL.x, toL.y, toL.z, __int_as_float(slot));
                    e.c = c;
                }
            }

            // PART 3: hero-wavelength BSDF sample (:4597-4719): cosine-weighted
            // direction, krayNM = reflectance(lambda), pdf = cos/pi.
            const float u1 = Rand(key, Dim(depth, 16)), u2 = Rand(key, Dim(depth, 17));
            const V3 w = dot(d, ns) > kNearZero ? -ns : ns;
            V3 tx, ty;
            Basis(w, tx, ty);
            const float phi = 2.0f * kPi * u1;
            const float sint = sqrtf(u2), cost = sqrtf(1.0f - u2);
            float sp, cp;
            __sincosf(phi, &sp, &cp);
            const V3 nd = normalize(tx * (cp * sint) + ty * (sp * sint) + w * cost);
            const float pdf = fabsf(dot(nd, w)) * kInvPi;
            // Geometric-horizon gate (LambertianSPF.cpp:141-151).
            const V3 gn = dot(ng, d) < 0.0f ? ng : -ng;
            if (!(dot(nd, gn) > 0.0f)) break;
            float4 kray;
            for (int k = 0; k < 4; ++k) Set(kray, k, (term & (1u << k)) ? 0.0f : Spec(S.spectra, M.refl, lam[k]));
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
                if (Rand(key, Dim(depth, 19)) >= prob) break;
                if (prob > 0.0f && prob < 1.0f) {
                    const float s = 1.0f / prob;
                    kray = make_float4(kray.x * s, kray.y * s, kray.z * s, kray.w * s);
                }
            }
            if (depth + 1 >= set.max_depth) break;
            thr = make_float4(thr.x * kray.x, thr.y * kray.y, thr.z * kray.z, thr.w * kray.w);
            const V3 no = OffsetRay(p, ng, nd);
            P.ray_o[slot] = make_float4(no.x, no.y, no.z, 0.0f);
            P.ray_d[slot] = make_float4(nd.x, nd.y, nd.z, __int_as_float(0x7f800000));
            P.thr[slot] = thr;
            P.aux[slot] = make_float4(aux.x, pdf, 0.0f, 0.0f);
            m.z = (m.z & ~kFlagDepthMask) | (unsigned)(depth + 1) | kFlagConsiderEmission;
            P.meta[slot].z = m.z;
            cont = true;
        } while (false);

        P.L[slot] = L;
        if (!cont) Finish(P, Q, slot, m, fin);
        const int an = WarpAppend(&Q.cnt[kCntActiveNext], cont);
        if (cont) Q.active_next[an] = slot;
        const int fn = WarpAppend(&Q.cnt[kCntFreeNext], fin);
        if (fin) Q.free_next[fn] = slot;
        // Shadow entries: lanes append their own count.
        {
            const unsigned act = __activemask();
            const int lane = threadIdx.x & 31;
            int incl = nsh;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(act, incl, o);
                if (lane >= o && ((act >> (lane - o)) & 1u)) incl += v;
            }
            const int leader = 31 - __clz(act);
            int base = 0;
            if (lane == leader && incl > 0) base = atomicAdd(&Q.cnt[kCntShadow], incl);
            base = __shfl_sync(act, base, leader);
            const int at0 = base + incl - nsh;
            for (int k = 0; k < nsh; ++k) Q.shadow[at0 + k] = sh[k];
        }
    }
}

__global__ void KSwap(int* cnt)
{
    cnt[kCntSegments] += cnt[kCntActive];
    cnt[kCntShadowRays] += cnt[kCntShadow];
    cnt[kCntActive] = cnt[kCntActiveNext];
    cnt[kCntActiveNext] = 0;
    cnt[kCntFree] = cnt[kCntFreeNext];
    cnt[kCntFreeNext] = 0;
    cnt[kCntShadow] = 0;
}

// Kahan-compensated fold of this call's film into the running sums.
__global__ void KFold(PtFilm F, int n3)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        const float y = F.pass[i] - F.comp[i];
        const float s = F.sum[i];
        const float t = s + y;
        F.comp[i] = (t - s) - y;
        F.sum[i] = t;
        F.pass[i] = 0.0f;
    }
}

// ---- host launcher ---------------------------------------------------------

namespace {
template <class K>
int TraceGrid(K kernel, int sms)
{
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kTraceBlock, 0) != cudaSuccess || per < 1) per = 1;
    return per * sms;
}
}  // namespace

cudaError_t PtIteration(const PtLaunch& L, cudaStream_t st)
{
    const int shadeGrid = L.sms * 8;
    KRegen<<<shadeGrid, kShadeBlock, 0, st>>>(L.paths, L.queues, L.film, L.params);
    cudaMemsetAsync(L.queues.trace_ctr, 0, 2 * sizeof(unsigned long long), st);
    if (L.scene.layout == RTB200_BVH_Q8) {
        static int g = 0;
        if (!g) g = TraceGrid(KExtend<QNode4>, L.sms);
        KExtend<QNode4><<<g, kTraceBlock, 0, st>>>((const QNode4*)L.scene.nodes, L.scene, L.paths, L.queues);
    } else {
        static int g = 0;
        if (!g) g = TraceGrid(KExtend<GpuNode4>, L.sms);
        KExtend<GpuNode4><<<g, kTraceBlock, 0, st>>>((const GpuNode4*)L.scene.nodes, L.scene, L.paths, L.queues);
    }
    KShade<<<shadeGrid, kShadeBlock, 0, st>>>(L.scene, L.paths, L.queues, L.params);
    if (L.scene.layout == RTB200_BVH_Q8) {
        static int g = 0;
        if (!g) g = TraceGrid(KConnect<QNode4>, L.sms);
        KConnect<QNode4><<<g, kTraceBlock, 0, st>>>((const QNode4*)L.scene.nodes, L.scene, L.paths, L.queues);
    } else {
        static int g = 0;
        if (!g) g = TraceGrid(KConnect<GpuNode4>, L.sms);
        KConnect<GpuNode4><<<g, kTraceBlock, 0, st>>>((const GpuNode4*)L.scene.nodes, L.scene, L.paths, L.queues);
    }
    KSwap<<<1, 1, 0, st>>>(L.queues.cnt);
    return cudaGetLastError();
}

cudaError_t PtFold(const PtFilm& F, int npix, int sms, cudaStream_t st)
{
    KFold<<<sms * 4, 256, 0, st>>>(F, 3 * npix);
    return cudaGetLastError();
}

}  // namespace rtb200
