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
//                E(mu_i)); the multiple-scattering lobe is sampled cosine-weighted.
//   Dielectric   DielectricSPF (Materials/DielectricSPF.cpp:120-451): smooth
//                interface, Fresnel-weighted choice between mirror reflection and
//                Snell refraction (delta lobes, no BSDF).
#pragma once
#include "pt_device.cuh"

namespace rtb200 {

constexpr int kLut = 32;
// E_ss / E_avg tables, uploaded at scene commit (defined here: this header is
// compiled into exactly one translation unit, pathtrace.cu).
__constant__ float c_ess[kLut * kLut];
__constant__ float c_eavg[kLut];

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
    const float v00 = c_ess[a0 * kLut + c0], v01 = c_ess[a0 * kLut + c1];
    const float v10 = c_ess[a1 * kLut + c0], v11 = c_ess[a1 * kLut + c1];
    return (1 - af) * ((1 - cf) * v00 + cf * v01) + af * ((1 - cf) * v10 + cf * v11);
}

__device__ __forceinline__ float LookupEavg(float alpha)
{
    const float a = fmaxf(0.0f, fminf(1.0f, (alpha - 0.01f) / 0.99f)) * (kLut - 1);
    const int a0 = (int)a;
    const int a1 = min(a0 + 1, kLut - 1);
    const float af = a - (float)a0;
    return (1 - af) * c_eavg[a0] + af * c_eavg[a1];
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
};

__device__ __forceinline__ GgxParams GgxAt(const PtMaterial& M, const float* spectra, float lam)
{
    GgxParams g;
    g.alpha = fmaxf(M.alpha, 1e-4f);
    g.spec = M.refl >= 0 ? Spec(spectra, M.refl, lam) : 1.0f;
    g.eta = M.eta >= 0 ? Spec(spectra, M.eta, lam) : M.ior;
    g.k = M.kappa >= 0 ? Spec(spectra, M.kappa, lam) : 0.0f;
    g.favg = M.pad >= 0 ? Spec(spectra, M.pad, lam) : 0.0f;
    return g;
}

// GGXBRDF::valueNM: r = towards the viewer, v = towards the light, n the
// shading normal on the viewer's side, gn the geometric normal facing the
// incoming ray.
__device__ __forceinline__ float GgxValue(const GgxParams& g, V3 n, V3 gn, V3 r, V3 v)
{
    const float nr = dot(n, r), nv = dot(n, v);
    if (nr < kNearZero || nv < kNearZero) return 0.0f;
    if (dot(v, gn) <= 0.0f || dot(r, gn) <= 0.0f) return 0.0f;
    const V3 h = normalize(v + r);
    const float D = GgxD(g.alpha, dot(h, n));
    const float G2 = 1.0f / (1.0f + GgxLambda(g.alpha, nv) + GgxLambda(g.alpha, nr));
    float f = 0.0f;
    const float sf = D * G2 / (4.0f * nv * nr);
    if (sf > 0.0f) f = g.spec * ConductorF(dot(r, h), 1.0f, g.eta, g.k) * sf;
    const float eavg = LookupEavg(g.alpha);
    if (1.0f - eavg > 1e-10f) {
        const float fm = (1.0f - LookupEss(nr, g.alpha)) * (1.0f - LookupEss(nv, g.alpha)) / (kPi * (1.0f - eavg));
        f += Fms(g.spec * g.favg, eavg) * fm;
    }
    return f;
}

// Mixture pdf of the GGX sampler at one wavelength (GGXSPF::Pdf); r towards
// the viewer, v the sampled direction.
__device__ __forceinline__ float GgxPdf(const GgxParams& g, V3 n, V3 gn, V3 r, V3 v)
{
    const float cosV = dot(v, n);
    if (cosV <= 0.0f || dot(v, gn) <= 0.0f) return 0.0f;
    const float ws = g.spec;
    const float wms = ws * (1.0f - LookupEss(dot(r, n), g.alpha));
    const float total = ws + wms;
    if (total <= 1e-10f) return 0.0f;
    return (wms * cosV * kInvPi + ws * VndfPdf(r, v, n, g.alpha)) / total;
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
