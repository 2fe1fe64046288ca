// env_map.h -- the image environment (a rasterizer's radiance_map bound to an
// HDR texture painter), shared by the host (importance-sampling tables) and
// the device (lookups, sampling, pdf).
//
// Restates, for this path:
//  * the light-probe (angular) mapping of RadianceMap::GetRadianceNM
//    (Rendering/RadianceMap.h) and EnvironmentSampler::DirectionToTexCoord /
//    TexCoordToDirection (Rendering/EnvironmentSampler.cpp): a map-space
//    direction v lands at s = 1/2 + v.x r, t = 1/2 - v.y r with
//    r = acos(-v.z) / (2 pi sqrt(v.x^2 + v.y^2));
//  * the bilinear texel lookup of BilinRasterImageAccessor::GetPel at the base
//    level (RasterImages/BilinRasterImageAccessor.h; rays carry no texture
//    footprint, so no mip level is chosen): column u = s W + 1/2 and row
//    v = t H + 1/2, clamped to the image, the four texels (floor, floor + 1)
//    clamped at the last row / column (the clamp-to-edge wrap mode);
//  * the per-lookup spectral uplift of TexturePainter::GetColorNM
//    (Painters/TexturePainter.cpp:200-240) for an HDR painter
//    (RGBUnboundedSpectrum, Utilities/Color/RGBSpectra.h:81-100): scale =
//    max channel, the sigmoid polynomial of rgb / scale from the Jakob-Hanika
//    table (zero polynomial below 1e-9), value = scale * sigmoid at lambda;
//  * EnvironmentSampler::Sample / Pdf: a 64 x 64 piecewise-constant density
//    over (s, t) -- row by the marginal CDF, column by the row's conditional
//    CDF, each by a binary search for the last entry <= the number -- turned
//    into a solid-angle density by theta / (4 pi^2 sin theta), theta = 2 pi
//    |(s, t) - (1/2, 1/2)|, with its limit 1 / (4 pi) near the centre or
//    outside the probe disk.
// The map's rotation (RadianceMap::SetOrientation: Euler angles) is applied
// to world directions before the mapping; sampled map directions go back
// through its transpose.
#pragma once

#include <cstdint>

#include "pt_types.h"

namespace rtb200 {

constexpr int kEnvCdfRes = 64;          // EnvironmentSampler resolution (RayCaster.cpp:346-351)
constexpr int kUpliftRes = 64;          // Jakob-Hanika table cells per axis

struct PtEnvMap {
    const float4* texels;       // width x height linear Rec.709 RGB, rows top to bottom (w unused)
    int width, height;
    float rot[9];               // world -> map, row major: map_i = sum_j rot[3 i + j] world_j
    float scale;                // radiance_scale
    const float* marginal;      // kEnvCdfRes + 1 entries, normalised
    const float* conditional;   // kEnvCdfRes rows of kEnvCdfRes + 1 entries, normalised
    const float* uplift;        // 3 x 64^3 cells of (c0, c1, c2): largest channel, z, x, y
};

RTB_HD void EnvProbeST(float x, float y, float z, float& s, float& t)
{
    const float den = sqrtf(x * x + y * y);
    if (den < 1e-12f) {
        s = 0.5f;
        t = 0.5f;
        return;
    }
    const float r = 0.159154943f * acosf(fmaxf(-1.0f, fminf(1.0f, -z))) / den;
    s = 0.5f + x * r;
    t = 0.5f - y * r;
}

RTB_HD void EnvProbeDir(float s, float t, float& x, float& y, float& z)
{
    const float dx = s - 0.5f, dy = -(t - 0.5f);
    const float rt = sqrtf(dx * dx + dy * dy);
    if (rt < 1e-12f) {
        x = 0.0f;
        y = 0.0f;
        z = -1.0f;
        return;
    }
    const float th = rt * 6.28318530717958647692f;
    const float st = sinf(th), ct = cosf(th);
    x = dx * st / rt;
    y = dy * st / rt;
    z = -ct;
}

// theta / (4 pi^2 sin theta) at (s, t), or 1 / (4 pi) at the centre and
// outside the disk; 0 where sin theta vanishes at the rim.
RTB_HD float EnvJacobian(float s, float t)
{
    const float dx = s - 0.5f, dy = -(t - 0.5f);
    const float rt = sqrtf(dx * dx + dy * dy);
    const float th = rt * 6.28318530717958647692f;
    if (th < 1e-6f || rt > 0.5f) return 0.0795774715f;
    const float st = sinf(th);
    if (st < 1e-10f) return 0.0f;
    return th / (39.4784176f * st);
}

RTB_HD float4 EnvTexel(const PtEnvMap& E, int x, int y)
{
#ifdef __CUDA_ARCH__
    return __ldg(E.texels + (size_t)y * E.width + x);
#else
    return E.texels[(size_t)y * E.width + x];
#endif
}

// BilinRasterImageAccessor::GetPel at (s, t) with clamp-to-edge.
RTB_HD void EnvBilinear(const PtEnvMap& E, float s, float t, float rgb[3])
{
    if (!(s == s) || !(t == t) || fabsf(s) > 1e30f || fabsf(t) > 1e30f) {
        rgb[0] = rgb[1] = rgb[2] = 0.0f;
        return;
    }
    float u = s * (float)E.width + 0.5f, v = t * (float)E.height + 0.5f;
    u = fminf(fmaxf(u, 0.0f), (float)(E.width - 1));
    v = fminf(fmaxf(v, 0.0f), (float)(E.height - 1));
    const float ulo = floorf(u), vlo = floorf(v);
    const float ut = u - ulo, vt = v - vlo;
    const int xlo = (int)ulo, ylo = (int)vlo;
    const int xhi = xlo + 1 >= E.width ? E.width - 1 : xlo + 1;
    const int yhi = ylo + 1 >= E.height ? E.height - 1 : ylo + 1;
    const float4 ll = EnvTexel(E, xlo, ylo), lh = EnvTexel(E, xhi, ylo), hl = EnvTexel(E, xlo, yhi),
                 hh = EnvTexel(E, xhi, yhi);
    const float a = (1.0f - ut) * (1.0f - vt), b = (1.0f - ut) * vt, c = ut * (1.0f - vt), d = ut * vt;
    rgb[0] = ll.x * a + hl.x * b + lh.x * c + hh.x * d;
    rgb[1] = ll.y * a + hl.y * b + lh.y * c + hh.y * d;
    rgb[2] = ll.z * a + hl.z * b + lh.z * c + hh.z * d;
}

// RGBToSpectrumTable's trilinear lookup of the sigmoid coefficients of an
// RGB in [0, 1] (the host's RgbToSigmoid in rgb_uplift.cpp, in FP32).
RTB_HD const float* UpliftCell(const float* T, int maxc, int iz, int ix, int iy)
{
    iz = iz < 0 ? 0 : (iz > kUpliftRes - 1 ? kUpliftRes - 1 : iz);
    ix = ix < 0 ? 0 : (ix > kUpliftRes - 1 ? kUpliftRes - 1 : ix);
    iy = iy < 0 ? 0 : (iy > kUpliftRes - 1 ? kUpliftRes - 1 : iy);
    return T + 3 * ((((size_t)maxc * kUpliftRes + iz) * kUpliftRes + ix) * kUpliftRes + iy);
}

RTB_HD void UpliftSigmoid(const float* T, float r, float g, float b, float c[3])
{
    r = fminf(fmaxf(r, 0.0f), 1.0f);
    g = fminf(fmaxf(g, 0.0f), 1.0f);
    b = fminf(fmaxf(b, 0.0f), 1.0f);
    int maxc;
    float z, x, y;
    if (r >= g && r >= b) {
        maxc = 0; z = r; x = z > 1e-9f ? g / z : 0.0f; y = z > 1e-9f ? b / z : 0.0f;
    } else if (g >= r && g >= b) {
        maxc = 1; z = g; x = z > 1e-9f ? b / z : 0.0f; y = z > 1e-9f ? r / z : 0.0f;
    } else {
        maxc = 2; z = b; x = z > 1e-9f ? r / z : 0.0f; y = z > 1e-9f ? g / z : 0.0f;
    }
    const float top = (float)(kUpliftRes - 1);
    const float fz = fminf(fmaxf(asinf(sqrtf(fminf(fmaxf(z, 0.0f), 1.0f))) * 0.636619772f * top, 0.0f), top);
    const float fx = fminf(fmaxf(x * top, 0.0f), top), fy = fminf(fmaxf(y * top, 0.0f), top);
    const int iz = (int)floorf(fz), ix = (int)floorf(fx), iy = (int)floorf(fy);
    const float tz = fz - (float)iz, tx = fx - (float)ix, ty = fy - (float)iy;
    for (int k = 0; k < 3; ++k) {
        const float c000 = UpliftCell(T, maxc, iz, ix, iy)[k], c010 = UpliftCell(T, maxc, iz, ix + 1, iy)[k];
        const float c100 = UpliftCell(T, maxc, iz + 1, ix, iy)[k], c110 = UpliftCell(T, maxc, iz + 1, ix + 1, iy)[k];
        const float c001 = UpliftCell(T, maxc, iz, ix, iy + 1)[k], c011 = UpliftCell(T, maxc, iz, ix + 1, iy + 1)[k];
        const float c101 = UpliftCell(T, maxc, iz + 1, ix, iy + 1)[k];
        const float c111 = UpliftCell(T, maxc, iz + 1, ix + 1, iy + 1)[k];
        const float a00 = c000 + (c010 - c000) * tx, a01 = c100 + (c110 - c100) * tx;
        const float a10 = c001 + (c011 - c001) * tx, a11 = c101 + (c111 - c101) * tx;
        const float b0 = a00 + (a10 - a00) * ty, b1 = a01 + (a11 - a01) * ty;
        c[k] = b0 + (b1 - b0) * tz;
    }
}

// The environment's radiance spectrum in a world direction: coefficients
// and scale of RGBUnboundedSpectrum (times radiance_scale); evaluate with
// EnvSpectrum.
struct EnvSpec {
    float c0, c1, c2, scale;
};

RTB_HD EnvSpec EnvLookup(const PtEnvMap& E, float wx, float wy, float wz)
{
    const float mx = E.rot[0] * wx + E.rot[1] * wy + E.rot[2] * wz;
    const float my = E.rot[3] * wx + E.rot[4] * wy + E.rot[5] * wz;
    const float mz = E.rot[6] * wx + E.rot[7] * wy + E.rot[8] * wz;
    float s, t, rgb[3];
    EnvProbeST(mx, my, mz, s, t);
    EnvBilinear(E, s, t, rgb);
    EnvSpec o{0.0f, 0.0f, 0.0f, 0.0f};
    const float m = fmaxf(rgb[0], fmaxf(rgb[1], rgb[2]));
    if (m > 1e-9f) {
        float c[3];
        UpliftSigmoid(E.uplift, rgb[0] / m, rgb[1] / m, rgb[2] / m, c);
        o.c0 = c[0];
        o.c1 = c[1];
        o.c2 = c[2];
    }
    o.scale = m * E.scale;
    return o;
}

RTB_HD float EnvSpectrum(const EnvSpec& e, float nm)
{
    if (nm < 380.0f || nm > 780.0f) return 0.0f;
    const float t = (nm - 380.0f) / 400.0f;
    const float x = e.c0 * t * t + e.c1 * t + e.c2;
    return e.scale * (0.5f + x / (2.0f * sqrtf(1.0f + x * x)));
}

// Largest i < n with cdf[i] <= xi (EnvironmentSampler::SampleCDF), and the
// fraction of xi within that bin.
RTB_HD int EnvSampleCdf(const float* cdf, int n, float xi, float& frac)
{
    int lo = 0, hi = n;
    while (lo + 1 < hi) {
        const int mid = (lo + hi) / 2;
        if (cdf[mid] <= xi) lo = mid;
        else hi = mid;
    }
    const float w = cdf[lo + 1] - cdf[lo];
    frac = w > 0.0f ? (xi - cdf[lo]) / w : 0.0f;
    return lo;
}

// EnvironmentSampler::Sample: a world direction and its solid-angle pdf
// (0 when the map is black).
RTB_HD float EnvSample(const PtEnvMap& E, float u1, float u2, float& wx, float& wy, float& wz)
{
    constexpr int R = kEnvCdfRes;
    float fv, fu;
    const int v = EnvSampleCdf(E.marginal, R, u2, fv);
    const float* row = E.conditional + (size_t)v * (R + 1);
    const int u = EnvSampleCdf(row, R, u1, fu);
    const float s = ((float)u + fu) / (float)R, t = ((float)v + fv) / (float)R;
    float mx, my, mz;
    EnvProbeDir(s, t, mx, my, mz);
    // Map -> world: the transpose of the rotation.
    wx = E.rot[0] * mx + E.rot[3] * my + E.rot[6] * mz;
    wy = E.rot[1] * mx + E.rot[4] * my + E.rot[7] * mz;
    wz = E.rot[2] * mx + E.rot[5] * my + E.rot[8] * mz;
    const float pst = (E.marginal[v + 1] - E.marginal[v]) * (float)R * (row[u + 1] - row[u]) * (float)R;
    return pst * EnvJacobian(s, t);
}

// EnvironmentSampler::Pdf of a world direction.
RTB_HD float EnvPdf(const PtEnvMap& E, float wx, float wy, float wz)
{
    constexpr int R = kEnvCdfRes;
    const float mx = E.rot[0] * wx + E.rot[1] * wy + E.rot[2] * wz;
    const float my = E.rot[3] * wx + E.rot[4] * wy + E.rot[5] * wz;
    const float mz = E.rot[6] * wx + E.rot[7] * wy + E.rot[8] * wz;
    float s, t;
    EnvProbeST(mx, my, mz, s, t);
    s = fmaxf(0.0f, fminf(0.999999f, s));
    t = fmaxf(0.0f, fminf(0.999999f, t));
    const int ui = (int)(s * (float)R), vi = (int)(t * (float)R);
    const int u = ui < R - 1 ? ui : R - 1, v = vi < R - 1 ? vi : R - 1;
    const float* row = E.conditional + (size_t)v * (R + 1);
    const float pst = (E.marginal[v + 1] - E.marginal[v]) * (float)R * (row[u + 1] - row[u]) * (float)R;
    return pst * EnvJacobian(s, t);
}

}  // namespace rtb200
