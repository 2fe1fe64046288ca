// pt_device.cuh -- device helpers of the spectral path tracer: counter-based
// random numbers, spectra and CIE lookups, HWSS wavelengths, small vector
// algebra, ray-origin offsetting, MIS weights and warp-aggregated appends.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "cie1931.h"
#include "pt_types.h"

namespace rtb200 {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kNearZero = 1e-12f;   // NEARZERO, Utilities/Math3D/Constants.h:33

// Defined here: this header is compiled into exactly one translation unit
// (pathtrace.cu).
__constant__ float c_cie[3][RTB200_CIE_COUNT] = {{RTB200_CIE_XBAR}, {RTB200_CIE_YBAR}, {RTB200_CIE_ZBAR}};

// ---- random numbers ---------------------------------------------------------
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
// uses 8 + 32*depth + j: light sample i at j = 4i..4i+3 (light, x, y,
// triangle), BSDF direction j = 16, 17, lobe / Fresnel choice 18, Russian
// roulette 19, sky sample i at j = 20 + 2i, 21 + 2i.
__device__ __forceinline__ uint32_t Dim(int depth, int j) { return 8u + 32u * (uint32_t)depth + (uint32_t)j; }

// ---- the reference's sampler: Owen-scrambled padded Sobol ------------------
// SobolSequence (Sampling/SobolSequence.h:55-206): dimension d of sample i is
// Sobol dimension d & 1 of i (dimension 0 the bit-reversed index, dimension 1
// the XOR of the direction numbers v_0 = 2^31, v_{k+1} = v_k ^ (v_k >> 1) over
// the set bits of i), Owen-scrambled by the Laine-Karras hash seeded with
// HashCombine(seed, d) (Burley 2020, "Practical Hash-based Owen Scrambling").

// HashCombine: a ^= b + golden + (a << 6) + (a >> 2), then MurmurHash3's
// fmix32 finaliser.
__device__ __forceinline__ uint32_t HashCombine(uint32_t a, uint32_t b)
{
    a ^= b + 0x9e3779b9u + (a << 6) + (a >> 2);
    a ^= a >> 16; a *= 0x85ebca6bu;
    a ^= a >> 13; a *= 0xc2b2ae35u;
    a ^= a >> 16;
    return a;
}

__device__ __forceinline__ uint32_t SobolDim1(uint32_t i)
{
    uint32_t v = 0, d = 1u << 31;
    while (i) {
        if (i & 1u) v ^= d;
        d ^= d >> 1;
        i >>= 1;
    }
    return v;
}

// Owen scrambling by the Laine-Karras hash on the bit-reversed value.
__device__ __forceinline__ uint32_t OwenScramble(uint32_t v, uint32_t s)
{
    v = __brev(v);
    v ^= v * 0x3d20adeau;
    v += s;
    v *= (s >> 16) | 1u;
    v ^= v * 0x05526c56u;
    v ^= v * 0x53a22864u;
    return __brev(v);
}

// shuffle: the sample index is first Owen-scrambled with a seed per
// dimension pair (2k, 2k + 1), Burley's decorrelation of padded dimensions
// ("Practical Hash-based Owen Scrambling", JCGT 9(4), 2020, section 4), so
// different pairs no longer replay one Sobol pair under another scramble;
// the reference pads without it.
__device__ __forceinline__ float SobolSample(uint32_t index, uint32_t dim, uint32_t seed, bool shuffle = false)
{
    if (shuffle) index = OwenScramble(index, HashCombine(HashCombine(seed, 0x5bd1e995u), dim >> 1));
    const uint32_t v = OwenScramble((dim & 1u) ? SobolDim1(index) : __brev(index), HashCombine(seed, dim));
    return (float)(v >> 8) * (1.0f / 16777216.0f);   // the top 24 bits: < 1 in FP32
}

// Sobol seed of a pixel: the reference's HashCombine(x, y); a nonzero job seed
// is mixed in so that renders with different seeds are independent.
__device__ __forceinline__ uint32_t SobolPixelSeed(uint32_t x, uint32_t y, uint32_t seed)
{
    const uint32_t s = HashCombine(x, y);
    return seed ? HashCombine(s, seed) : s;
}

// Random numbers of one path vertex.  Hash mode: Rand(key, Dim(depth, j))
// with the fixed layout above.  Sobol mode: the reference's
// StartStream(16 + depth) then dimensions in the order they are drawn
// (`cur`), so each call site names its hash-layout slot j and the Sobol
// dimension follows the draw order; skip(n) consumes dimensions that the
// reference draws but this vertex does not use.
struct VertexRng {
    uint32_t key;      // hash key, or the pixel's Sobol seed
    uint32_t index;    // sample index (Sobol)
    int depth;
    int mode;          // kSamplerHash / kSamplerSobol / kSamplerSobolShuffled
    uint32_t cur;
    __device__ __forceinline__ float next(int j)
    {
        if (mode != kSamplerHash)
            return SobolSample(index, (16u + (uint32_t)depth) * 32u + cur++, key, mode == kSamplerSobolShuffled);
        return Rand(key, Dim(depth, j));
    }
    __device__ __forceinline__ void skip(int n) { cur += (uint32_t)n; }
};

// ---- spectra -----------------------------------------------------------------

// Spectrum table: one float4 header per spectrum id, then the samples.
// Header {0, 380, 780, offset}: 81 samples on the 5 nm grid, linear between
// them (InterpSPDIndices, src/Library/Utilities/Color/ColorUtils.cpp:270-300),
// 0 outside 380..780 nm.  Header {n, begin, end, offset}: a binned packet of
// n amplitudes over [begin, end], the bin holding nm returned as is, 0
// outside (SpectralPacket::ValueAtNM, Utilities/Color/SpectralPacket.h:285-297;
// nm == end reads the last bin).  Header {-1, 380, 780, offset}: an RGB
// colour's sigmoid polynomial (c0, c1, c2, scale), scale * s(c0 t^2 + c1 t +
// c2) with t = (nm - 380) / 400 (RGBSigmoidPolynomial::Eval,
// Utilities/Color/RGBSigmoidPolynomial.h:58-70).  Header {-2, 0, 1e30,
// offset}: a black body (temperature, scale): scale * C1 / l^5 /
// (exp(C2 / (l T)) - 1) with l = nm * 1e-9 m, C1 = 2 pi h c^2, C2 = h c / k
// (BlackBodyPainter::GetColorNM, Painters/BlackBodyPainter.cpp:26-43,103-106).
// offset is the samples' float index (bits).
__device__ __forceinline__ float Spec(const float* table, int id, float nm)
{
    if (id < 0) return 0.0f;
    const float4 h = __ldg(reinterpret_cast<const float4*>(table) + id);
    const float* s = table + __float_as_int(h.w);
    if (!(nm >= h.y) || nm > h.z) return 0.0f;
    if (h.x == -2.0f) {
        // C1 / l^5 with l in nm: 2 pi h c^2 * 1e45 / nm^5; C2 / (l T) = h c / k * 1e9 / (nm T).
        const float T = __ldg(s), k = __ldg(s + 1);
        const float n2 = nm * nm;
        const float first = 3.7417749e29f / (n2 * n2 * nm);
        return k * first / (expf(1.4387687e7f / (nm * T)) - 1.0f);
    }
    if (h.x < 0.0f) {
        const float4 c = make_float4(__ldg(s), __ldg(s + 1), __ldg(s + 2), __ldg(s + 3));
        const float t = (nm - 380.0f) / 400.0f;
        const float x = c.x * t * t + c.y * t + c.z;
        return c.w * (0.5f + x / (2.0f * sqrtf(1.0f + x * x)));
    }
    if (h.x == 0.0f) {
        const float x = (nm - 380.0f) * 0.2f;
        const int i = (int)floorf(x);
        const int j = i + 1 > 80 ? 80 : i + 1;
        const float w = x - (float)i;
        return __ldg(s + i) + w * (__ldg(s + j) - __ldg(s + i));
    }
    const int n = (int)h.x;
    const int i = min((int)((nm - h.y) * h.x / (h.z - h.y)), n - 1);
    return __ldg(s + i);
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

// ---- small vector helpers ---------------------------------------------------

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

// Unit vector from its octahedral encoding (OctEncode in pt_types.h).
__device__ __forceinline__ V3 OctDecode(unsigned q)
{
    const float u = (float)(short)(q & 0xffffu) * (1.0f / 32767.0f);
    const float v = (float)(short)(q >> 16) * (1.0f / 32767.0f);
    float x = u, y = v;
    const float z = 1.0f - fabsf(u) - fabsf(v);
    if (z < 0.0f) {
        x = (1.0f - fabsf(v)) * (u >= 0.0f ? 1.0f : -1.0f);
        y = (1.0f - fabsf(u)) * (v >= 0.0f ? 1.0f : -1.0f);
    }
    return normalize(mk(x, y, z));
}

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

// Warp-aggregated queue append: one atomic per warp; returns this lane's
// index (or -1 when `pred` is false).
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

}  // namespace rtb200
