// bsdf.cuh -- material models of the spectral path tracer (device side).
//
//   Lambertian   LambertianSPF / LambertianBRDF (Materials/LambertianSPF.cpp:90-172,
//                LambertianBRDF.cpp:44-93): cosine sampling, f = rho/pi.
//   GGX          GGXSPF / GGXBRDF conductor mode (Materials/GGXSPF.cpp:424-688,
//                GGXBRDF.cpp:339-498): specular lobe with visible-normal sampling
//                (spherical caps, Dupuy and Benyoub 2023), height-correlated Smith
//                G2, unpolarised conductor Fresnel (Utilities/Optics.hpp), plus the
//                Kulla-Conty multiple-scattering lobe F_ms (1-E(mu_o))(1-E(mu_i)) /
//                (pi (1-E_avg)) (Utilities/MicrofacetEnergyLUT.h).  Lobes are picked
//                with the reference's weights w_s = specular colour, w_ms = w_s (1 -
//                E(mu_i)); the multiple-scattering lobe samples mu_o from its own
//                shape (1 - E(mu_o)) mu_o by exact inversion of the piecewise-cubic
//                CDF, with the matching density (MicrofacetEnergyLUT.h:122-333).
//   Dielectric   DielectricSPF (Materials/DielectricSPF.cpp:120-451): smooth
//                interface, Fresnel-weighted choice between mirror reflection and
//                Snell refraction (delta lobes, no BSDF).
#pragma once
#include "pt_device.cuh"

namespace rtb200 {

constexpr int kLut = 32;
// Energy tables, uploaded at the first scene commit (defined here: this header
// is compiled into exactly one translation unit, pathtrace.cu).  They live in
// global memory and are read through the read-only cache: lanes of a warp
// shade different materials and roughnesses, and divergent indices would
// serialise constant-memory reads.
__device__ float g_ess[kLut * kLut];          // E_ss[alpha row][mu cell]
__device__ float g_eavg[kLut];
__device__ float g_msz[kLut];                 // per row: 2 * integral of (1 - E_ss(mu)) mu dmu
__device__ float g_mscum[kLut * (kLut + 2)];  // per row: integral of the lobe shape up to each segment
constexpr int kFavgNodes = 21;
__device__ float g_favg_x[kFavgNodes];        // Gauss-Legendre nodes on [0, 1] and weights 2 mu w
__device__ float g_favg_w[kFavgNodes];

// MicrofacetEnergyLUT::LookupEss / LookupEavg (MicrofacetEnergyLUT.h:90-120):
// bilinear in (alpha, mu) with mu at cell centres.
__device__ __forceinline__ float LookupEss(float cosT, float alpha)
{
    const float a = fmaxf(0.0f, fminf(1.0f, (alpha - 0.01f) / 0.99f)) * (kLut - 1);
    const int a0 = (int)a;
    const int a1 = min(a0 + 1, kLut - 1);
    const float af = a - (float)a0;
    float c = fmaxf(0.0f, fminf(1.0f, cosT)) * kLut - 0.5f;
    if (c < 0.0f) c = 0.0f;
    const int c0 = (int)c;
    const int c1 = min(c0 + 1, kLut - 1);
    const float cf = c - (float)c0;
    const float v00 = __ldg(g_ess + a0 * kLut + c0), v01 = __ldg(g_ess + a0 * kLut + c1);
    const float v10 = __ldg(g_ess + a1 * kLut + c0), v11 = __ldg(g_ess + a1 * kLut + c1);
    return (1 - af) * ((1 - cf) * v00 + cf * v01) + af * ((1 - cf) * v10 + cf * v11);
}

__device__ __forceinline__ float LookupEavg(float alpha)
{
    const float a = fmaxf(0.0f, fminf(1.0f, (alpha - 0.01f) / 0.99f)) * (kLut - 1);
    const int a0 = (int)a;
    const int a1 = min(a0 + 1, kLut - 1);
    const float af = a - (float)a0;
    return (1 - af) * __ldg(g_eavg + a0) + af * __ldg(g_eavg + a1);
}

__device__ __forceinline__ void AlphaRow(float alpha, int& a0, int& a1, float& af)
{
    const float a = fmaxf(0.0f, fminf(1.0f, (alpha - 0.01f) / 0.99f)) * (kLut - 1);
    a0 = (int)a;
    a1 = min(a0 + 1, kLut - 1);
    af = a - (float)a0;
}

// Normalisation Z(alpha) of the multiple-scattering lobe shape (1 - E(mu)) mu
// (MSLobeZ): exact per table row, linear in the row blend.
__device__ __forceinline__ float MsZ(float alpha)
{
    int a0, a1;
    float af;
    AlphaRow(alpha, a0, a1, af);
    return (1.0f - af) * __ldg(g_msz + a0) + af * __ldg(g_msz + a1);
}

// Solid-angle density of the multiple-scattering lobe sampler (MSPdf).
__device__ __forceinline__ float MsPdf(float c, float alpha, float z)
{
    if (z <= 1e-15f) return 0.0f;
    c = fmaxf(0.0f, fminf(1.0f, c));
    return fmaxf(0.0f, (1.0f - LookupEss(c, alpha)) * c / (kPi * z));
}

// Segment k (0 .. kLut) of the alpha-blended piecewise-linear E(mu): flat caps
// below the first and above the last cell centre, linear spans between.
struct MsSeg {
    float lo, w, e0, slope;
};

__device__ __forceinline__ MsSeg MsSegment(int a0, int a1, float af, int k)
{
    MsSeg s;
    const int j0 = max(k - 1, 0), j1 = min(k, kLut - 1);
    const float r0 = (1.0f - af) * __ldg(g_ess + a0 * kLut + j0) + af * __ldg(g_ess + a1 * kLut + j0);
    const float r1 = (1.0f - af) * __ldg(g_ess + a0 * kLut + j1) + af * __ldg(g_ess + a1 * kLut + j1);
    s.lo = k == 0 ? 0.0f : (k - 0.5f) / kLut;
    s.w = (k == 0 || k == kLut) ? 0.5f / kLut : 1.0f / kLut;
    s.e0 = k == 0 ? r1 : r0;
    s.slope = (k == 0 || k == kLut) ? 0.0f : (r1 - r0) * kLut;
    return s;
}

// Integral of the lobe shape over the first y of a segment.
__device__ __forceinline__ float MsCdf(const MsSeg& s, float y)
{
    const float P = (1.0f - s.e0) * s.lo, Q = (1.0f - s.e0) - s.slope * s.lo, R = -s.slope;
    return y * (P + y * (0.5f * Q + y * (R * (1.0f / 3.0f))));
}

// Integral of the lobe shape over segments 0 .. k-1 of the blended row.  The
// segment integrals are linear in the row values, hence in the row blend, so
// the per-row cumulative tables blend exactly like E_ss itself.
__device__ __forceinline__ float MsCum(int a0, int a1, float af, int k)
{
    return (1.0f - af) * __ldg(g_mscum + a0 * (kLut + 2) + k) + af * __ldg(g_mscum + a1 * (kLut + 2) + k);
}

// mu_o for the multiple-scattering lobe from one uniform number
// (SampleMSCosTheta): find the segment whose cumulative integral brackets
// u * I (binary search over the 33 segments), then invert its cubic CDF by
// Newton steps kept inside a bisection bracket.
__device__ __forceinline__ float MsSampleCos(float alpha, float u)
{
    int a0, a1;
    float af;
    AlphaRow(alpha, a0, a1, af);
    const float I = MsCum(a0, a1, af, kLut + 1);
    if (!(I > 1e-15f)) return fmaxf(0.0f, fminf(1.0f, u));
    const float target = fmaxf(0.0f, fminf(I, u * I));
    // Largest k in [0, kLut] with cum(k) < target (segment k holds the target).
    int lo_k = 0, hi_k = kLut;
    while (lo_k < hi_k) {
        const int mid = (lo_k + hi_k + 1) >> 1;
        if (MsCum(a0, a1, af, mid) < target) lo_k = mid; else hi_k = mid - 1;
    }
    const int k = lo_k;
    const MsSeg s = MsSegment(a0, a1, af, k);
    const float run = MsCum(a0, a1, af, k);
    const float tot = MsCdf(s, s.w);
    const float goal = fmaxf(0.0f, fminf(tot, target - run));
    float lo = 0.0f, hi = s.w, y = 0.5f * s.w;
    for (int it = 0; it < 30; ++it) {
        const float diff = MsCdf(s, y) - goal;
        if (fabsf(diff) <= 1e-7f * tot) break;
        if (diff > 0.0f) hi = y; else lo = y;
        const float dv = fmaxf(0.0f, (1.0f - (s.e0 + s.slope * y)) * (s.lo + y));
        float nx = dv > 1e-12f ? y - diff / dv : 0.5f * (lo + hi);
        if (!(nx > lo && nx < hi)) nx = 0.5f * (lo + hi);
        y = nx;
    }
    return fmaxf(0.0f, fminf(1.0f, s.lo + y));
}

__device__ __forceinline__ float GgxLambda(float alpha, float cosT)
{
    if (cosT >= 1.0f - 1e-7f) return 0.0f;
    if (cosT < 1e-10f) return 1e10f;
    const float c2 = cosT * cosT;
    const float t2 = (1.0f - c2) / c2;
    return (-1.0f + sqrtf(1.0f + alpha * alpha * t2)) * 0.5f;
}

__device__ __forceinline__ float GgxD(float alpha, float cosH)
{
    if (cosH <= 0.0f) return 0.0f;
    const float a2 = alpha * alpha;
    const float d = cosH * cosH * (a2 - 1.0f) + 1.0f;
    return a2 / (kPi * d * d);
}

// Visible-normal pdf of reflecting wi into wo (MicrofacetUtils VNDF_Pdf).
__device__ __forceinline__ float VndfPdf(V3 wi, V3 wo, V3 n, float alpha)
{
    const float cosI = dot(wi, n);
    if (cosI < 1e-10f) return 0.0f;
    const V3 h = normalize(wi + wo);
    const float ch = dot(h, n), ih = dot(wi, h), oh = dot(wo, h);
    if (ch <= 0.0f || ih <= 0.0f || oh < 1e-10f) return 0.0f;
    const float g1 = 1.0f / (1.0f + GgxLambda(alpha, cosI));
    return g1 * ih * GgxD(alpha, ch) / cosI / (4.0f * oh);
}

// Unpolarised conductor Fresnel reflectance (Optics.hpp CalculateConductorReflectance).
__device__ __forceinline__ float ConductorF(float cosI, float ni, float nt, float kt)
{
    float c = fabsf(cosI);
    if (c < 1e-12f) c = 1e-12f;
    const float c2 = c * c;
    const float s2 = fmaxf(0.0f, 1.0f - c2);
    const float s = sqrtf(s2);
    const float tn = s / c;
    const float ni2 = ni * ni, nt2 = nt * nt, k2 = kt * kt;
    const float ns = ni2 * s2, nk = 4.0f * nt2 * k2;
    float a2 = nt2 - k2 - ns;
    const float sq = sqrtf(a2 * a2 + nk);
    float b2 = sq - nt2 + k2 + ns;
    a2 = sq + nt2 - k2 - ns;
    const float dni = 0.5f / ni2;
    a2 = fmaxf(0.0f, a2 * dni);
    b2 = fmaxf(0.0f, b2 * dni);
    const float a = sqrtf(a2);
    const float ab2 = a2 + b2;
    const float dcos = 2.0f * a * c;
    const float astan = 2.0f * a * s * tn;
    const float stan = s2 * tn * tn;
    const float rs = (ab2 - dcos + c2) / (ab2 + dcos + c2);
    const float rp = rs * (ab2 - astan + stan) / (ab2 + astan + stan);
    return 0.5f * (rp + rs);
}

// MicrofacetEnergyLUT::ComputeFms (MicrofacetEnergyLUT.h:407-425).
__device__ __forceinline__ float Fms(float favg, float eavg)
{
    const float den = 1.0f - favg * (1.0f - eavg);
    return den < 1e-10f ? 0.0f : favg * favg * eavg / den;
}

struct GgxParams {
    float alpha;
    float spec;    // specular colour at this wavelength
    float eta, k;  // conductor optical constants
    float favg;    // hemispherical average of the conductor Fresnel
    float amb;     // index of the medium around the surface (1: air)
};

// Hemispherical average 2 * integral of F(mu) mu dmu of the conductor
// Fresnel from a medium of index ni (MicrofacetEnergyLUT::ComputeFresnelAvg,
// 21-point Gauss-Legendre); only paths inside a dielectric need it, air's is
// a spectrum of the material.
__device__ __noinline__ float ConductorFavg(float ni, float nt, float kt)
{
    float s = 0.0f;
    #pragma unroll 1
    for (int i = 0; i < kFavgNodes; ++i) s += ConductorF(__ldg(g_favg_x + i), ni, nt, kt) * __ldg(g_favg_w + i);
    return s;
}

// One wavelength's parameters from the values a shading point looked up once
// for each of its wavelengths (specular colour, optical constants, and the
// Fresnel average for the incident index amb: GgxFavg).  amb is the index of
// the medium around the hit, the top of the path's index-of-refraction stack,
// which the conductor Fresnel takes as the incident index (GGXBRDF.cpp:430-434).
__device__ __forceinline__ GgxParams GgxFrom(const PtMaterial& M, float spec, float eta, float k, float favg, float amb)
{
    GgxParams g;
    g.alpha = fmaxf(M.alpha, 1e-4f);
    g.spec = spec;
    g.eta = eta;
    g.k = k;
    g.favg = favg;
    g.amb = amb;
    return g;
}

// The conductor's hemispherical Fresnel average at one wavelength for the
// incident index amb (GGXBRDF.cpp:476-481): air's is a spectrum of the
// material, any other is integrated here.
__device__ __forceinline__ float GgxFavg(const PtMaterial& M, const float* spectra, float lam, float amb, float eta,
                                         float k)
{
    if (amb == 1.0f) return M.pad >= 0 ? Spec(spectra, M.pad, lam) : 0.0f;
    return ConductorFavg(amb, eta, k);
}

// ---- evaluation split by what depends on the wavelength ----------------------
// Roughness is the same at every wavelength, so the microfacet terms, the
// energy-table lookups and the sampling density are computed once per shading
// point or direction pair; only the Fresnel terms and the specular colour are
// evaluated per wavelength.  The pair and per-wavelength evaluations are
// called from several places in the shading kernel and kept out of line: the
// inlined copies overflowed the instruction cache (ncu: stalls on
// no_instruction dominated; out of line and with the per-wavelength loops not
// unrolled the GGX/glass scene renders 10 % faster).

// Per shading point: E_ss at the viewer direction, E_avg and the
// multiple-scattering lobe normalisation.
struct GgxPoint {
    float alpha, essR, eavg, msz;
};

__device__ __forceinline__ GgxPoint GgxPointAt(float alpha, float cosR)
{
    GgxPoint g;
    g.alpha = fmaxf(alpha, 1e-4f);
    g.essR = LookupEss(cosR, g.alpha);
    g.eavg = LookupEavg(g.alpha);
    g.msz = MsZ(g.alpha);
    return g;
}

// Per (viewer r, light v) pair: the single-scattering factor D G2 / (4 nv nr)
// and Fresnel cosine, the multiple-scattering factor (1-E(nr))(1-E(nv)) /
// (pi (1-E_avg)), and the sampling density, which does not depend on the
// specular colour (the lobe weights w_s and w_s (1 - E(nr)) share it).
struct GgxPair {
    float sf, rh, ms, pdf;
    bool ok;
};

__device__ __noinline__ GgxPair GgxPairAt(const GgxPoint& g, V3 n, V3 gn, V3 r, V3 v)
{
    GgxPair q;
    q.sf = q.rh = q.ms = q.pdf = 0.0f;
    const float nr = dot(n, r), nv = dot(n, v);
    q.ok = nr >= kNearZero && nv >= kNearZero && dot(v, gn) > 0.0f && dot(r, gn) > 0.0f;
    if (!q.ok) return q;
    const V3 h = normalize(v + r);
    const float ch = dot(h, n);
    const float D = GgxD(g.alpha, ch);
    const float lr = GgxLambda(g.alpha, nr);
    const float G2 = 1.0f / (1.0f + GgxLambda(g.alpha, nv) + lr);
    q.sf = D * G2 / (4.0f * nv * nr);
    q.rh = dot(r, h);
    const float essV = LookupEss(nv, g.alpha);
    if (1.0f - g.eavg > 1e-10f) q.ms = (1.0f - g.essR) * (1.0f - essV) / (kPi * (1.0f - g.eavg));
    // VNDF pdf of reflecting r into v (MicrofacetUtils VNDF_Pdf).
    const float oh = dot(v, h);
    float vndf = 0.0f;
    if (nr >= 1e-10f && ch > 0.0f && q.rh > 0.0f && oh >= 1e-10f)
        vndf = (1.0f / (1.0f + lr)) * q.rh * D / nr / (4.0f * oh);
    const float mspdf = g.msz <= 1e-15f ? 0.0f : fmaxf(0.0f, (1.0f - essV) * fminf(nv, 1.0f) / (kPi * g.msz));
    q.pdf = ((1.0f - g.essR) * mspdf + vndf) / (2.0f - g.essR);
    return q;
}

// The BSDF at one wavelength for a pair (GGXBRDF::valueNM).
__device__ __noinline__ float GgxValueAt(const GgxPair& q, const GgxParams& p, float eavg)
{
    if (!q.ok) return 0.0f;
    float f = 0.0f;
    if (q.sf > 0.0f) f = p.spec * ConductorF(q.rh, p.amb, p.eta, p.k) * q.sf;
    return f + Fms(p.spec * p.favg, eavg) * q.ms;
}

// Visible-normal sample around n for the view direction r (local frame
// t, b, n): the reference's spherical-cap construction (MicrofacetUtils.h).
__device__ __forceinline__ V3 VndfSample(V3 r, V3 t, V3 b, V3 n, float alpha, float u1, float u2)
{
    const V3 wl = mk(dot(r, t), dot(r, b), dot(r, n));
    const V3 wh = normalize(mk(alpha * wl.x, alpha * wl.y, wl.z));
    const float phi = 2.0f * kPi * u1;
    const float z = (1.0f - u2) * (1.0f + wh.z) - wh.z;
    const float st = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float sp, cp;
    __sincosf(phi, &sp, &cp);
    const V3 c = mk(st * cp + wh.x, st * sp + wh.y, z + wh.z);
    const V3 ml = normalize(mk(alpha * c.x, alpha * c.y, c.z));
    return normalize(t * ml.x + b * ml.y + n * ml.z);
}

// Dielectric Fresnel reflectance for unit incident and transmitted directions
// (Optics::CalculateDielectricReflectance, Utilities/Optics.cpp:101-160).
__device__ __forceinline__ float DielectricR(float cosI, float cosT, float ni, float nt)
{
    const float nn = ni * nt, cc = cosT * cosI;
    const float ni2 = ni * ni, nt2 = nt * nt;
    const float ci2 = cosI * cosI, ct2 = cosT * cosT;
    const float nit = ni2 - nt2, cit = ci2 - ct2;
    const float num = nit * nit * cc * cc + cit * cit * nn * nn;
    float den = cc * (ni2 + nt2) + nn * (ci2 + ct2);
    den = den * den;
    if (den < 1e-6f && num < 1e-6f) return 1.0f;
    return fminf(1.0f, num / den);
}

}  // namespace rtb200
