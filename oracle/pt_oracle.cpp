// pt_oracle.cpp -- TEST INFRASTRUCTURE ONLY (oracle port).
//
// Double-precision, one-sample-at-a-time restatement of the reference's
// hero-wavelength spectral path tracer for the scenes of this project
// (triangle meshes; Lambertian, GGX-conductor and smooth-dielectric
// materials; Lambertian area emitters; uniform sky):
//   * per-pixel sample loop, box pixel filter   PathTracingSpectralRasterizer.cpp:206-479
//   * 4 equidistant wavelengths, XYZ, (b-a)/k_y  PathTracingSpectralRasterizer.cpp:121-198,
//                                                SampledWavelengths.h:79-106,
//                                                ColorUtils.cpp:270-348
//   * bounce loop                               PathTracingIntegrator.cpp:4094-4817
//       runaway guard :4099-4110, emission + MIS :4424-4518, NEE per
//       wavelength :4523-4550, BSDF sample + companions :4597-4719,
//       Russian roulette :4738-4769, update + Advance(1e-8) :4791-4816
//   * area-light and sky NEE                    LightSampler.cpp:2083-2359
//   * Lambertian                                LambertianSPF.cpp:90-172, LambertianBRDF.cpp:44-93,
//                                                GeometricUtilities.cpp:85-98
//   * GGX conductor                             GGXSPF.cpp:424-688, GGXBRDF.cpp:339-498,
//                                                MicrofacetUtils.h, MicrofacetEnergyLUT.h, Optics.hpp
//   * smooth dielectric                         DielectricSPF.cpp:120-300, :395-432, Optics.cpp:39-160
//   * index-of-refraction stack per path         IORStack.h, PathTracingIntegrator.cpp:4315-4328,
//                                                :4684, :4814-4816; conductor incident index
//                                                GGXBRDF.cpp:430-434, :476-481
//   * point on a mesh luminary                  TriangleMeshGeometryIndexed.cpp:207-218,
//                                                GeometricUtilities.cpp:543-569
//   * power heuristic, Russian roulette         PathTransportUtilities.h:86-110, :251
// Random numbers come from the same samplers the device has (the counter-
// based hash, the reference's Owen-scrambled Sobol and its shuffled variant),
// so a pixel sample follows the same decisions here and on the GPU up to
// rounding.
// Loaded only by tests and bench.py's CPU-baseline leg.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

const double kPi = 3.14159265358979323846;
const double kInvPi = 1.0 / kPi;
const double kInv4Pi = 1.0 / (4.0 * kPi);
const double kNearZero = 1e-12;

inline uint32_t Mix32(uint32_t x)
{
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
inline uint32_t PathKey(uint32_t seed, uint32_t pixel, uint32_t sample)
{
    return Mix32(Mix32(seed ^ 0x9e3779b9u ^ Mix32(pixel)) ^ sample);
}
inline double Rand(uint32_t key, uint32_t dim)
{
    return (double)(Mix32(key ^ (dim * 0x9e3779b9u + 0x7f4a7c15u)) >> 8) * (1.0 / 16777216.0);
}
inline uint32_t Dim(int depth, int j) { return 8u + 32u * (uint32_t)depth + (uint32_t)j; }

// The reference's sampler (Sampling/SobolSequence.h:55-206,
// Utilities/SobolSampler.h): padded Owen-scrambled Sobol.
inline uint32_t HashCombine(uint32_t a, uint32_t b)
{
    a ^= b + 0x9e3779b9u + (a << 6) + (a >> 2);
    a ^= a >> 16; a *= 0x85ebca6bu;
    a ^= a >> 13; a *= 0xc2b2ae35u;
    a ^= a >> 16;
    return a;
}
inline uint32_t ReverseBits(uint32_t n)
{
    n = (n << 16) | (n >> 16);
    n = ((n & 0x00ff00ffu) << 8) | ((n & 0xff00ff00u) >> 8);
    n = ((n & 0x0f0f0f0fu) << 4) | ((n & 0xf0f0f0f0u) >> 4);
    n = ((n & 0x33333333u) << 2) | ((n & 0xccccccccu) >> 2);
    n = ((n & 0x55555555u) << 1) | ((n & 0xaaaaaaaau) >> 1);
    return n;
}
inline uint32_t SobolBits(uint32_t index, uint32_t dim, uint32_t seed)
{
    uint32_t v = 0;
    if (dim & 1u) {
        for (uint32_t i = index, d = 1u << 31; i; i >>= 1, d ^= d >> 1)
            if (i & 1u) v ^= d;
    } else {
        v = ReverseBits(index);
    }
    const uint32_t s = HashCombine(seed, dim);
    v = ReverseBits(v);
    v ^= v * 0x3d20adeau;
    v += s;
    v *= (s >> 16) | 1u;
    v ^= v * 0x05526c56u;
    v ^= v * 0x53a22864u;
    return ReverseBits(v);
}
inline uint32_t OwenScrambleBits(uint32_t v, uint32_t s)
{
    v = ReverseBits(v);
    v ^= v * 0x3d20adeau;
    v += s;
    v *= (s >> 16) | 1u;
    v ^= v * 0x05526c56u;
    v ^= v * 0x53a22864u;
    return ReverseBits(v);
}
// As the device draws it: the top 24 bits; shuffle: the index first
// Owen-scrambled with a seed per dimension pair (Burley, JCGT 9(4), 2020).
inline double SobolSample(uint32_t index, uint32_t dim, uint32_t seed, bool shuffle = false)
{
    if (shuffle) index = OwenScrambleBits(index, HashCombine(HashCombine(seed, 0x5bd1e995u), dim >> 1));
    return (double)(SobolBits(index, dim, seed) >> 8) * (1.0 / 16777216.0);
}
inline uint32_t SobolPixelSeed(uint32_t x, uint32_t y, uint32_t seed)
{
    const uint32_t s = HashCombine(x, y);
    return seed ? HashCombine(s, seed) : s;
}

// Numbers of one path vertex: the fixed hash layout, or the reference's
// StartStream(16 + depth) and dimensions in draw order (the device's
// VertexRng).
struct VertexRng {
    uint32_t key, index;
    int depth;
    int mode;          // 0 hash, 1 Sobol, 2 Sobol with shuffled indices
    uint32_t cur;
    double next(int j)
    {
        if (mode) return SobolSample(index, (16u + (uint32_t)depth) * 32u + cur++, key, mode == 2);
        return Rand(key, Dim(depth, j));
    }
    void skip(int n) { cur += (uint32_t)n; }
};

struct V { double x, y, z; };
inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator*(V a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V operator-(V a) { return {-a.x, -a.y, -a.z}; }
inline double Dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V Cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V Norm(V a) { return a * (1.0 / std::sqrt(Dot(a, a))); }

// Frame around unit n (Duff et al., JCGT 6(1), 2017) -- the device's frame,
// so that equal random numbers give equal directions.
inline void Frame(V n, V& t, V& b)
{
    const double sg = std::copysign(1.0, n.z);
    const double a = -1.0 / (sg + n.z);
    const double c = n.x * n.y * a;
    t = {1.0 + sg * n.x * n.x * a, sg * c, -sg * n.x};
    b = {c, sg + n.y * n.y * a, -n.y};
}

// ---- GGX conductor ----------------------------------------------------------

double Lambda(double alpha, double c)
{
    if (c >= 1.0 - 1e-10) return 0.0;
    if (c < 1e-10) return 1e10;
    const double c2 = c * c;
    return (-1.0 + std::sqrt(1.0 + alpha * alpha * (1.0 - c2) / c2)) * 0.5;
}
double GgxD(double alpha, double ch)
{
    if (ch <= 0) return 0.0;
    const double a2 = alpha * alpha;
    const double d = ch * ch * (a2 - 1.0) + 1.0;
    return a2 / (kPi * d * d);
}
// Spherical-cap visible-normal sample for view direction wl (local frame).
V VndfLocal(V wl, double alpha, double u1, double u2)
{
    const V wh = Norm({alpha * wl.x, alpha * wl.y, wl.z});
    const double phi = 2.0 * kPi * u1;
    const double z = (1.0 - u2) * (1.0 + wh.z) - wh.z;
    const double st = std::sqrt(std::max(0.0, 1.0 - z * z));
    const V c = {st * std::cos(phi) + wh.x, st * std::sin(phi) + wh.y, z + wh.z};
    return Norm({alpha * c.x, alpha * c.y, c.z});
}
double VndfPdf(V wi, V wo, V n, double alpha)
{
    const double ci = Dot(wi, n);
    if (ci < 1e-10) return 0.0;
    const V h = Norm(wi + wo);
    const double ch = Dot(h, n), ih = Dot(wi, h), oh = Dot(wo, h);
    if (ch <= 0 || ih <= 0 || oh < 1e-10) return 0.0;
    const double g1 = 1.0 / (1.0 + Lambda(alpha, ci));
    return g1 * ih * GgxD(alpha, ch) / ci / (4.0 * oh);
}
double ConductorF(double cosI, double ni, double nt, double kt)
{
    double c = std::fabs(cosI);
    if (c < 1e-12) c = 1e-12;
    const double c2 = c * c, s2 = std::max(0.0, 1.0 - c2), s = std::sqrt(s2), tn = s / c;
    const double ni2 = ni * ni, nt2 = nt * nt, k2 = kt * kt, ns = ni2 * s2, nk = 4.0 * nt2 * k2;
    double a2 = nt2 - k2 - ns;
    const double sq = std::sqrt(a2 * a2 + nk);
    double b2 = sq - nt2 + k2 + ns;
    a2 = sq + nt2 - k2 - ns;
    const double dni = 0.5 / ni2;
    a2 = std::max(0.0, a2 * dni);
    b2 = std::max(0.0, b2 * dni);
    const double a = std::sqrt(a2), ab2 = a2 + b2, dcos = 2.0 * a * c, astan = 2.0 * a * s * tn, stan = s2 * tn * tn;
    const double rs = (ab2 - dcos + c2) / (ab2 + dcos + c2);
    const double rp = rs * (ab2 - astan + stan) / (ab2 + astan + stan);
    return 0.5 * (rp + rs);
}

struct Tables {
    double ess[32][32];
    double eavg[32];
    double msz[32];   // multiple-scattering lobe normalisation per alpha row
    double glx[21], glw[21];
};

void ComputeMsZ(Tables& T);
int kEssStrata = 128;   // strata per axis of each E_ss cell

Tables& MutableTables()
{
    static Tables T;
    static std::once_flag once;
    std::call_once(once, []() {
        // Gauss-Legendre nodes on [0, 1].
        const int n = 21;
        for (int i = 0; i < n; ++i) {
            double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
            for (int it = 0; it < 100; ++it) {
                double p0 = 1.0, p1 = z;
                for (int k = 2; k <= n; ++k) { const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = p2; }
                const double dp = n * (z * p1 - p0) / (z * z - 1.0);
                const double dz = p1 / dp;
                z -= dz;
                if (std::fabs(dz) < 1e-15) break;
            }
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) { const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = p2; }
            const double dp = n * (z * p1 - p0) / (z * z - 1.0);
            T.glx[i] = 0.5 * (z + 1.0);
            T.glw[i] = 1.0 / ((1.0 - z * z) * dp * dp);
        }
        // E_ss(mu, alpha) by stratified visible-normal integration of the
        // reference table's estimator (tools/GenerateMicrofacetEnergyLUT.cpp:
        // reflect the view direction about a visible normal, weight by the
        // masking G1 of the reflected direction), and E_avg by its midpoint
        // sum 2 * sum(E_ss mu) / 32.
        for (int a = 0; a < 32; ++a) {
            const double alpha = 0.01 + 0.99 * a / 31.0;
            double avg = 0.0;
            for (int c = 0; c < 32; ++c) {
                const double mu = (c + 0.5) / 32.0;
                const V wo = {std::sqrt(std::max(0.0, 1.0 - mu * mu)), 0.0, mu};
                const int ns = kEssStrata;
                double sum = 0.0;
                for (int i = 0; i < ns; ++i)
                    for (int j = 0; j < ns; ++j) {
                        const V m = VndfLocal(wo, alpha, (i + 0.5) / ns, (j + 0.5) / ns);
                        const double d = Dot(wo, m);
                        if (d <= 0) continue;
                        const V wi = Norm(m * (2.0 * d) - wo);
                        if (wi.z <= 0) continue;
                        sum += 1.0 / (1.0 + Lambda(alpha, wi.z));
                    }
                T.ess[a][c] = sum / ((double)ns * ns);
                avg += T.ess[a][c] * mu;
            }
            T.eavg[a] = 2.0 * avg / 32.0;
        }
        ComputeMsZ(T);
    });
    return T;
}
const Tables& GetTables() { return MutableTables(); }

double LookupEss(double cosT, double alpha)
{
    const Tables& T = GetTables();
    const double a = std::max(0.0, std::min(1.0, (alpha - 0.01) / 0.99)) * 31.0;
    const int a0 = (int)a, a1 = std::min(a0 + 1, 31);
    const double af = a - a0;
    double c = std::max(0.0, std::min(1.0, cosT)) * 32.0 - 0.5;
    if (c < 0) c = 0;
    const int c0 = (int)c, c1 = std::min(c0 + 1, 31);
    const double cf = c - c0;
    return (1 - af) * ((1 - cf) * T.ess[a0][c0] + cf * T.ess[a0][c1]) + af * ((1 - cf) * T.ess[a1][c0] + cf * T.ess[a1][c1]);
}
double LookupEavg(double alpha)
{
    const Tables& T = GetTables();
    const double a = std::max(0.0, std::min(1.0, (alpha - 0.01) / 0.99)) * 31.0;
    const int a0 = (int)a, a1 = std::min(a0 + 1, 31);
    const double af = a - a0;
    return (1 - af) * T.eavg[a0] + af * T.eavg[a1];
}
// ---- multiple-scattering lobe sampler (MicrofacetEnergyLUT.h:122-333) --------
// E_ss is piecewise linear in mu between bin centres (flat outside the first
// and last centre), so the lobe shape (1 - E_ss(mu)) mu is piecewise quadratic:
// 33 segments with a closed-form cubic CDF, inverted by Newton steps kept
// inside a bisection bracket.
struct MsSeg { double lo, hi, e0, slope; };

void MsSegments(const double row[32], MsSeg seg[33])
{
    seg[0] = {0.0, 0.5 / 32.0, row[0], 0.0};
    for (int k = 0; k < 31; ++k) {
        const double a = (k + 0.5) / 32.0, b = (k + 1.5) / 32.0;
        seg[k + 1] = {a, b, row[k], (row[k + 1] - row[k]) / (b - a)};
    }
    seg[32] = {31.5 / 32.0, 1.0, row[31], 0.0};
}
double MsShape(const MsSeg& s, double y) { return std::max(0.0, (1.0 - (s.e0 + s.slope * y)) * (s.lo + y)); }
double MsCdf(const MsSeg& s, double y)
{
    const double P = (1.0 - s.e0) * s.lo, Q = (1.0 - s.e0) - s.slope * s.lo, R = -s.slope;
    return P * y + Q * y * y * 0.5 + R * y * y * y * (1.0 / 3.0);
}
double MsInvert(const MsSeg& s, double target, double w)
{
    double lo = 0.0, hi = w, y = 0.5 * w;
    for (int it = 0; it < 30; ++it) {
        const double diff = MsCdf(s, y) - target;
        if (std::fabs(diff) < 1e-13) break;
        if (diff > 0) hi = y; else lo = y;
        const double dv = MsShape(s, y);
        double nx = dv > 1e-12 ? y - diff / dv : 0.5 * (lo + hi);
        if (!(nx > lo && nx < hi)) nx = 0.5 * (lo + hi);
        y = nx;
    }
    return y;
}
void AlphaRow(double alpha, int& a0, int& a1, double& af)
{
    const double a = std::max(0.0, std::min(1.0, (alpha - 0.01) / 0.99)) * 31.0;
    a0 = (int)a;
    a1 = std::min(a0 + 1, 31);
    af = a - a0;
}
void ComputeMsZ(Tables& T)
{
    for (int r = 0; r < 32; ++r) {
        MsSeg seg[33];
        MsSegments(T.ess[r], seg);
        double I = 0.0;
        for (const MsSeg& s : seg) I += MsCdf(s, s.hi - s.lo);
        T.msz[r] = 2.0 * I;
    }
}
double MsZ(double alpha)
{
    const Tables& T = GetTables();
    int a0, a1;
    double af;
    AlphaRow(alpha, a0, a1, af);
    return (1.0 - af) * T.msz[a0] + af * T.msz[a1];
}
double MsPdf(double c, double alpha, double z)
{
    if (z <= 1e-15) return 0.0;
    c = std::max(0.0, std::min(1.0, c));
    return std::max(0.0, (1.0 - LookupEss(c, alpha)) * c / (kPi * z));
}
double MsSampleCos(double alpha, double u)
{
    const Tables& T = GetTables();
    int a0, a1;
    double af;
    AlphaRow(alpha, a0, a1, af);
    double row[32];
    for (int k = 0; k < 32; ++k) row[k] = (1.0 - af) * T.ess[a0][k] + af * T.ess[a1][k];
    MsSeg seg[33];
    MsSegments(row, seg);
    double tot[33], I = 0.0;
    for (int k = 0; k < 33; ++k) { tot[k] = MsCdf(seg[k], seg[k].hi - seg[k].lo); I += tot[k]; }
    if (I <= 1e-15) return std::max(0.0, std::min(1.0, u));
    const double target = std::max(0.0, std::min(I, u * I));
    int k = 0;
    double run = 0.0;
    while (k < 32 && run + tot[k] < target) { run += tot[k]; ++k; }
    const double y = MsInvert(seg[k], std::max(0.0, std::min(tot[k], target - run)), seg[k].hi - seg[k].lo);
    return std::max(0.0, std::min(1.0, seg[k].lo + y));
}

double FresnelAvg(double ni, double nt, double kt)
{
    const Tables& T = GetTables();
    double s = 0.0;
    for (int i = 0; i < 21; ++i) s += ConductorF(T.glx[i], ni, nt, kt) * 2.0 * T.glx[i] * T.glw[i];
    return s;
}
double Fms(double favg, double eavg)
{
    const double den = 1.0 - favg * (1.0 - eavg);
    return den < 1e-10 ? 0.0 : favg * favg * eavg / den;
}

struct Ggx { double alpha, spec, eta, k, favg, amb; };

struct Light {
    int first, count, emit;
    double area, pdf;
    int bvhPos = 0;
    int kind = 0;      // 1: point light at pos with flat luminance le
    double le = 0.0;
    V pos = {0, 0, 0};
};

// Light BVH (Lights/LightBVH.cpp:132-531): preorder nodes over the
// luminaries, the left child after its parent.
struct LightNode {
    double lo[3], hi[3], power;
    int right = 0, light = -1, count = 0, start = 0;
};
struct LightPrimD {
    double lo[3], hi[3], c[3], power;
    int light;
};

// BuildRecursive (LightBVH.cpp:291-421): union box and summed power; split
// on the widest axis of the box centres at the power-weighted mean centre.
int BuildLightBvh(std::vector<LightPrimD>& prims, int start, int end, int& pos, std::vector<LightNode>& nodes,
                  std::vector<int>& posOf)
{
    const int idx = (int)nodes.size();
    nodes.emplace_back();
    LightNode n;
    n.power = prims[start].power;
    for (int k = 0; k < 3; ++k) { n.lo[k] = prims[start].lo[k]; n.hi[k] = prims[start].hi[k]; }
    for (int i = start + 1; i < end; ++i) {
        for (int k = 0; k < 3; ++k) { n.lo[k] = std::min(n.lo[k], prims[i].lo[k]); n.hi[k] = std::max(n.hi[k], prims[i].hi[k]); }
        n.power += prims[i].power;
    }
    n.count = end - start;
    n.start = pos;
    if (end - start == 1) {
        n.light = prims[start].light;
        posOf[n.light] = pos++;
        nodes[idx] = n;
        return idx;
    }
    double clo[3], chi[3];
    for (int k = 0; k < 3; ++k) clo[k] = chi[k] = prims[start].c[k];
    for (int i = start + 1; i < end; ++i)
        for (int k = 0; k < 3; ++k) { clo[k] = std::min(clo[k], prims[i].c[k]); chi[k] = std::max(chi[k], prims[i].c[k]); }
    const double ex[3] = {chi[0] - clo[0], chi[1] - clo[1], chi[2] - clo[2]};
    int axis = 0;
    if (ex[1] > ex[0]) axis = 1;
    if (ex[2] > (axis == 0 ? ex[0] : ex[1])) axis = 2;
    int mid;
    if (ex[axis] < 1e-10) {
        mid = start + (end - start) / 2;
    } else {
        double ws = 0.0, tp = 0.0;
        for (int i = start; i < end; ++i) { ws += prims[i].c[axis] * prims[i].power; tp += prims[i].power; }
        const double split = tp > 0.0 ? ws / tp : 0.5 * (clo[axis] + chi[axis]);
        auto it = std::partition(prims.begin() + start, prims.begin() + end,
                                 [&](const LightPrimD& p) { return p.c[axis] < split; });
        mid = (int)(it - prims.begin());
        if (mid == start || mid == end) mid = start + (end - start) / 2;
    }
    nodes[idx] = n;
    BuildLightBvh(prims, start, mid, pos, nodes, posOf);
    nodes[idx].right = (int)nodes.size();
    BuildLightBvh(prims, mid, end, pos, nodes, posOf);
    return idx;
}

// NodeImportance (LightBVH.cpp:169-217), full-sphere cone.
double LightImportance(const LightNode& n, const double p[3])
{
    if (!(n.power > 0)) return 0.0;
    double d2 = 0.0;
    for (int k = 0; k < 3; ++k) {
        const double d = p[k] < n.lo[k] ? n.lo[k] - p[k] : (p[k] > n.hi[k] ? p[k] - n.hi[k] : 0.0);
        d2 += d * d;
    }
    return n.power / std::max(d2, 1e-4);
}

// Sample (LightBVH.cpp:423-482): -1 with pdf 0 when nothing can be picked.
int SampleLightBvh(const std::vector<LightNode>& nodes, const double p[3], double xi, double& pdf)
{
    pdf = 1.0;
    int i = 0;
    while (nodes[i].count > 1) {
        const int r = nodes[i].right;
        const double il = LightImportance(nodes[i + 1], p), ir = LightImportance(nodes[r], p), tot = il + ir;
        if (!(tot > 0)) { pdf = 0.0; return -1; }
        const double pl = il / tot;
        if (xi < pl) { pdf *= pl; xi = xi / pl; i = i + 1; }
        else { pdf *= 1.0 - pl; xi = (xi - pl) / (1.0 - pl); i = r; }
    }
    return nodes[i].light;
}

// Pdf (LightBVH.cpp:484-531).
double LightBvhPdf(const std::vector<LightNode>& nodes, int pos, const double p[3])
{
    double pdf = 1.0;
    int i = 0;
    while (nodes[i].count > 1) {
        const int r = nodes[i].right;
        const double il = LightImportance(nodes[i + 1], p), ir = LightImportance(nodes[r], p), tot = il + ir;
        if (!(tot > 0)) return 0.0;
        const double pl = il / tot;
        const LightNode& L = nodes[i + 1];
        if (pos >= L.start && pos < L.start + L.count) { pdf *= pl; i = i + 1; }
        else { pdf *= 1.0 - pl; i = r; }
    }
    return pdf;
}
struct LTri { V v0, e1, e2; double cdf; };

// Octahedral unit-vector encoding as the device stores vertex normals
// (Cigolle et al., JCGT 3(2), 2014; OctEncode, rise_b200/csrc/pt_types.h):
// FP32 encode, decode back to a unit vector.
inline unsigned OctEncode(float x, float y, float z)
{
    const float s = std::fabs(x) + std::fabs(y) + std::fabs(z);
    float u = s > 0.0f ? x / s : 0.0f, v = s > 0.0f ? y / s : 0.0f;
    if (z < 0.0f) {
        const float fu = (1.0f - std::fabs(v)) * (u >= 0.0f ? 1.0f : -1.0f);
        const float fv = (1.0f - std::fabs(u)) * (v >= 0.0f ? 1.0f : -1.0f);
        u = fu;
        v = fv;
    }
    const int qu = (int)std::rint(std::fmin(std::fmax(u, -1.0f), 1.0f) * 32767.0f);
    const int qv = (int)std::rint(std::fmin(std::fmax(v, -1.0f), 1.0f) * 32767.0f);
    return ((unsigned)qu & 0xffffu) | ((unsigned)qv << 16);
}

// The image environment (a radiance_map bound to an HDR texture painter),
// restated in FP64: Rendering/RadianceMap.h (light-probe mapping, rotation
// XRotation * YRotation * ZRotation applied as Vector3Ops::Transform),
// RasterImages/BilinRasterImageAccessor.h GetPel (u = s W + 1/2, v = t H +
// 1/2, clamp to edge), Painters/TexturePainter.cpp:200-240 with
// Utilities/Color/RGBSpectra.h:81-100 (unbounded uplift per lookup from the
// Jakob-Hanika table, RGBToSpectrumTable.cpp:161-243), and
// Rendering/EnvironmentSampler.cpp (64 x 64 tables weighted by max channel x
// sin(theta) / theta, Sample / Pdf with theta / (4 pi^2 sin theta)).
struct EnvImage {
    const float* rgb = nullptr;   // w x h x 3, rows top to bottom
    int w = 0, h = 0;
    double scale = 1.0;
    double rot[3][3];             // world -> map: map_i = sum_j rot[i][j] world_j
    const float* table = nullptr; // 3 x 64^3 x 3 sigmoid coefficients
    std::vector<double> marg, cond;   // 65, 64 x 65

    void Rotation(const double o[3])
    {
        // Matrix4 storage _rc, XRotation / YRotation / ZRotation, product
        // ret._rc = sum_k a._kc b._rk, Transform out_c = sum_r m._rc v_r.
        auto ident = [](double m[4][4]) {
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j) m[i][j] = i == j;
        };
        double X[4][4], Y[4][4], Z[4][4];
        ident(X); ident(Y); ident(Z);
        X[1][1] = std::cos(o[0]); X[1][2] = std::sin(o[0]); X[2][1] = -std::sin(o[0]); X[2][2] = std::cos(o[0]);
        Y[2][2] = std::cos(o[1]); Y[2][0] = std::sin(o[1]); Y[0][2] = -std::sin(o[1]); Y[0][0] = std::cos(o[1]);
        Z[0][0] = std::cos(o[2]); Z[0][1] = std::sin(o[2]); Z[1][0] = -std::sin(o[2]); Z[1][1] = std::cos(o[2]);
        auto mul = [](const double a[4][4], const double b[4][4], double r[4][4]) {
            for (int rr = 0; rr < 4; ++rr)
                for (int c = 0; c < 4; ++c) {
                    double t = 0;
                    for (int k = 0; k < 4; ++k) t += a[k][c] * b[rr][k];
                    r[rr][c] = t;
                }
        };
        double XY[4][4], M[4][4];
        mul(X, Y, XY);
        mul(XY, Z, M);
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) rot[c][r] = M[r][c];
    }
    void Bilinear(double s, double t, double out[3]) const
    {
        if (!std::isfinite(s) || !std::isfinite(t)) { out[0] = out[1] = out[2] = 0; return; }
        double u = std::min(std::max(s * w + 0.5, 0.0), (double)(w - 1));
        double v = std::min(std::max(t * h + 0.5, 0.0), (double)(h - 1));
        const double ulo = std::floor(u), vlo = std::floor(v), ut = u - ulo, vt = v - vlo;
        const int xlo = (int)ulo, ylo = (int)vlo, xhi = std::min(xlo + 1, w - 1), yhi = std::min(ylo + 1, h - 1);
        auto px = [&](int x, int y, int k) { return (double)rgb[3 * ((size_t)y * w + x) + k]; };
        for (int k = 0; k < 3; ++k)
            out[k] = px(xlo, ylo, k) * ((1 - ut) * (1 - vt)) + px(xlo, yhi, k) * ((1 - ut) * vt) +
                     px(xhi, ylo, k) * (ut * (1 - vt)) + px(xhi, yhi, k) * (ut * vt);
    }
    static void ProbeST(const double m[3], double& s, double& t)
    {
        const double den = std::sqrt(m[0] * m[0] + m[1] * m[1]);
        if (den < 1e-12) { s = t = 0.5; return; }
        const double r = 0.159154943 * std::acos(std::max(-1.0, std::min(1.0, -m[2]))) / den;
        s = 0.5 + m[0] * r;
        t = 0.5 - m[1] * r;
    }
    static double Jacobian(double s, double t)
    {
        const double dx = s - 0.5, dy = -(t - 0.5), rt = std::sqrt(dx * dx + dy * dy), th = rt * 2 * kPi;
        if (th < 1e-6 || rt > 0.5) return 1.0 / (4 * kPi);
        const double st = std::sin(th);
        if (st < 1e-10) return 0.0;
        return th / (4 * kPi * kPi * st);
    }
    void ToMap(V d, double m[3]) const
    {
        const double w3[3] = {d.x, d.y, d.z};
        for (int i = 0; i < 3; ++i) m[i] = rot[i][0] * w3[0] + rot[i][1] * w3[1] + rot[i][2] * w3[2];
    }
    // Coefficients and scale of the radiance spectrum in world direction d.
    void Lookup(V d, double c[3], double& sc) const
    {
        double m[3], s, t, px[3];
        ToMap(d, m);
        ProbeST(m, s, t);
        Bilinear(s, t, px);
        const double mx = std::max(px[0], std::max(px[1], px[2]));
        c[0] = c[1] = c[2] = 0.0;
        if (mx > 1e-9) Uplift(px[0] / mx, px[1] / mx, px[2] / mx, c);
        sc = mx * scale;
    }
    void Uplift(double r, double g, double b, double c[3]) const
    {
        constexpr int R = 64;
        r = std::min(std::max(r, 0.0), 1.0); g = std::min(std::max(g, 0.0), 1.0); b = std::min(std::max(b, 0.0), 1.0);
        int mc; double z, x, y;
        if (r >= g && r >= b) { mc = 0; z = r; x = z > 1e-9 ? g / z : 0; y = z > 1e-9 ? b / z : 0; }
        else if (g >= r && g >= b) { mc = 1; z = g; x = z > 1e-9 ? b / z : 0; y = z > 1e-9 ? r / z : 0; }
        else { mc = 2; z = b; x = z > 1e-9 ? r / z : 0; y = z > 1e-9 ? g / z : 0; }
        const double fz = std::min(std::max(std::asin(std::sqrt(std::min(std::max(z, 0.0), 1.0))) * (2 / kPi) * (R - 1), 0.0), (double)(R - 1));
        const double fx = std::min(std::max(x * (R - 1), 0.0), (double)(R - 1)), fy = std::min(std::max(y * (R - 1), 0.0), (double)(R - 1));
        const int iz = (int)fz, ix = (int)fx, iy = (int)fy;
        const double tz = fz - iz, tx = fx - ix, ty = fy - iy;
        auto cell = [&](int zz, int xx, int yy, int k) {
            zz = std::min(zz, R - 1); xx = std::min(xx, R - 1); yy = std::min(yy, R - 1);
            return (double)table[3 * ((((size_t)mc * R + zz) * R + xx) * R + yy) + k];
        };
        for (int k = 0; k < 3; ++k) {
            const double a00 = cell(iz, ix, iy, k) + (cell(iz, ix + 1, iy, k) - cell(iz, ix, iy, k)) * tx;
            const double a01 = cell(iz + 1, ix, iy, k) + (cell(iz + 1, ix + 1, iy, k) - cell(iz + 1, ix, iy, k)) * tx;
            const double a10 = cell(iz, ix, iy + 1, k) + (cell(iz, ix + 1, iy + 1, k) - cell(iz, ix, iy + 1, k)) * tx;
            const double a11 = cell(iz + 1, ix, iy + 1, k) + (cell(iz + 1, ix + 1, iy + 1, k) - cell(iz + 1, ix, iy + 1, k)) * tx;
            const double b0 = a00 + (a10 - a00) * ty, b1 = a01 + (a11 - a01) * ty;
            c[k] = b0 + (b1 - b0) * tz;
        }
    }
    static double Spectrum(const double c[3], double sc, double nm)
    {
        if (nm < 380.0 || nm > 780.0) return 0.0;
        const double t = (nm - 380.0) / 400.0, x = c[0] * t * t + c[1] * t + c[2];
        return sc * (0.5 + x / (2.0 * std::sqrt(1.0 + x * x)));
    }
    void Build()
    {
        constexpr int R = 64;
        cond.assign((size_t)R * (R + 1), 0.0);
        marg.assign(R + 1, 0.0);
        for (int v = 0; v < R; ++v) {
            double* row = &cond[(size_t)v * (R + 1)];
            for (int u = 0; u < R; ++u) {
                const double s = (u + 0.5) / R, t = (v + 0.5) / R;
                double px[3];
                Bilinear(s, t, px);
                const double lum = std::max(px[0], std::max(px[1], px[2])) * scale;
                const double dx = s - 0.5, dy = -(t - 0.5), rt = std::sqrt(dx * dx + dy * dy), th = rt * 2 * kPi;
                double wgt = th < 1e-6 ? 1.0 : std::sin(th) / th;
                if (rt > 0.5) wgt = 0.0;
                row[u + 1] = row[u] + lum * wgt;
            }
        }
        for (int v = 0; v < R; ++v) marg[v + 1] = marg[v] + cond[(size_t)v * (R + 1) + R];
        const double tot = marg[R];
        if (!(tot > 0)) return;
        for (int v = 0; v < R; ++v) {
            double* row = &cond[(size_t)v * (R + 1)];
            const double rt = row[R];
            if (rt > 0)
                for (int u = 0; u <= R; ++u) row[u] /= rt;
            row[R] = 1.0;
        }
        for (double& m : marg) m /= tot;
        marg[R] = 1.0;
    }
    static int SampleCdf(const double* cdf, int n, double xi, double& frac)
    {
        int lo = 0, hi = n;
        while (lo + 1 < hi) {
            const int mid = (lo + hi) / 2;
            if (cdf[mid] <= xi) lo = mid; else hi = mid;
        }
        const double wd = cdf[lo + 1] - cdf[lo];
        frac = wd > 0 ? (xi - cdf[lo]) / wd : 0.0;
        return lo;
    }
    double Sample(double u1, double u2, V& d) const
    {
        constexpr int R = 64;
        double fv, fu;
        const int v = SampleCdf(marg.data(), R, u2, fv);
        const double* row = &cond[(size_t)v * (R + 1)];
        const int u = SampleCdf(row, R, u1, fu);
        const double s = (u + fu) / R, t = (v + fv) / R;
        const double dx = s - 0.5, dy = -(t - 0.5), rt = std::sqrt(dx * dx + dy * dy);
        double m[3] = {0, 0, -1};
        if (rt >= 1e-12) {
            const double th = rt * 2 * kPi;
            m[0] = dx * std::sin(th) / rt;
            m[1] = dy * std::sin(th) / rt;
            m[2] = -std::cos(th);
        }
        d = {rot[0][0] * m[0] + rot[1][0] * m[1] + rot[2][0] * m[2], rot[0][1] * m[0] + rot[1][1] * m[1] + rot[2][1] * m[2],
             rot[0][2] * m[0] + rot[1][2] * m[1] + rot[2][2] * m[2]};
        return (marg[v + 1] - marg[v]) * R * (row[u + 1] - row[u]) * R * Jacobian(s, t);
    }
    double Pdf(V d) const
    {
        constexpr int R = 64;
        double m[3], s, t;
        ToMap(d, m);
        ProbeST(m, s, t);
        s = std::max(0.0, std::min(0.999999, s));
        t = std::max(0.0, std::min(0.999999, t));
        const int u = std::min((int)(s * R), R - 1), v = std::min((int)(t * R), R - 1);
        const double* row = &cond[(size_t)v * (R + 1)];
        return (marg[v + 1] - marg[v]) * R * (row[u + 1] - row[u]) * R * Jacobian(s, t);
    }
};

struct Scene {
    EnvImage envImg;                       // used when envImg.rgb is set
    const float* tri9;
    const float* nrm9 = nullptr;           // vertex normals per triangle corner, or null (face normals)
    std::vector<unsigned> octN;            // their encodings, 3 per triangle (all zero: a flat triangle)
    std::vector<int> triMesh;
    const int64_t* meshes;
    const float* spectra;
    const int32_t* mi;
    const float* mf;
    const double* cie;
    std::vector<Light> lights;
    std::vector<double> aliasProb;         // alias table over the luminaries (power selection)
    std::vector<int> aliasOf;
    std::vector<LTri> ltris;
    std::vector<int> meshLight;
    orc_bvh* bvh;
    int env, envVisible;
    double lmin, lmax, rrThreshold, ynorm;
    int width, height, maxDepth, rrMinDepth, neePerLambda;
    int sampler = 0;                       // 0 hash, 1 Sobol, 2 Sobol with shuffled indices
    int maxBounce[3] = {255, 255, 255};    // diffuse, glossy, transmission
    int single = 0;                        // one wavelength per path (IntegrateRayNM)
    int numWl = 0;                         // single: wavelength bins (0 = continuous)
    double wlStep = 0.0;                   // single: (lmax - lmin) / numWl
    int spectral = 1;                      // paths per pixel sample (nSpectralSamples)
    uint32_t seed;
    bool lightBvh = false;                 // luminaries picked with the light BVH
    std::vector<LightNode> lightNodes;
    V pos, fwd, right, up;
    // Gaussian pixel filter too narrow for the filtered film: the camera
    // sample is warped about the pixel centre (warpSigma > 0), else 0.
    double warpSigma = 0.0, warpTrunc = 1.0;
};

// InterpSPDIndices + linear interpolation (ColorUtils.cpp:270-300).
inline bool Interp(double nm, int& i, int& j, double& w)
{
    if (nm < 380.0 || nm > 780.0) return false;
    const double x = (nm - 380.0) / 5.0;
    i = (int)std::floor(x);
    j = std::min(i + 1, 80);
    w = x - i;
    return true;
}
// Spectrum table: per id a header of 4 floats, {0, 380, 780, offset} for 81
// samples on the 5 nm grid (linear between them), {n, begin, end, offset}
// for a binned packet (SpectralPacket::ValueAtNM,
// Utilities/Color/SpectralPacket.h:285-297: the amplitude of bin
// int((nm - begin) / delta), delta = (end - begin) / n, 0 outside; nm == end
// reads the last bin); offset is the samples' float index (bits).
struct SpecHeader {
    double n, begin, end;
    const float* s;
};
// BlackBodyPainter::GetColorNM (Painters/BlackBodyPainter.cpp:26-43,103-106):
// scale * Planck's function of nm * 1e-9 m; s = (temperature, scale).
inline double Blackbody(const float* s, double nm)
{
    const double c = 2.99792458e8, h = 6.6260755e-34, k = 1.380658e-23;
    const double c1 = 2.0 * kPi * h * (c * c), c2 = (h * c) / k;
    const double lam = nm * 1e-9, t = s[0];
    return (double)s[1] * (c1 / std::pow(lam, 5.0) * (1.0 / (std::exp(c2 / (lam * t)) - 1.0)));
}

inline SpecHeader Header(const float* table, int id)
{
    const float* h = table + 4 * (size_t)id;
    int32_t off;
    std::memcpy(&off, h + 3, 4);
    return {h[0], h[1], h[2], table + off};
}
inline double Spec(const Scene& S, int id, double nm)
{
    if (id < 0) return 0.0;
    const SpecHeader h = Header(S.spectra, id);
    if (h.n == -2.0) return Blackbody(h.s, nm);
    if (h.n < 0.0) {
        // RGBSigmoidPolynomial::Eval (Utilities/Color/RGBSigmoidPolynomial.h:58-70) x scale.
        if (nm < 380.0 || nm > 780.0) return 0.0;
        const double t = (nm - 380.0) / 400.0;
        const double x = (double)h.s[0] * t * t + (double)h.s[1] * t + (double)h.s[2];
        return (double)h.s[3] * (0.5 + x / (2.0 * std::sqrt(1.0 + x * x)));
    }
    if (h.n == 0.0) {
        int i, j;
        double w;
        if (!Interp(nm, i, j, w)) return 0.0;
        return (double)h.s[i] + w * ((double)h.s[j] - (double)h.s[i]);
    }
    if (nm < h.begin || nm > h.end) return 0.0;
    const double delta = (h.end - h.begin) / h.n;
    return (double)h.s[std::min((int)((nm - h.begin) / delta), (int)h.n - 1)];
}
// The spectrum at grid point k (380 + 5k nm) as the scene upload tabulates it.
inline double GridValue(const float* table, int id, int k)
{
    const SpecHeader h = Header(table, id);
    if (h.n == -2.0) return (float)Blackbody(h.s, 380.0 + 5.0 * k);
    if (h.n < 0.0) {
        const double t = (5.0 * k) / 400.0;
        const double x = (double)h.s[0] * t * t + (double)h.s[1] * t + (double)h.s[2];
        return (float)((double)h.s[3] * (0.5 + x / (2.0 * std::sqrt(1.0 + x * x))));
    }
    if (h.n == 0.0) return h.s[k];
    const double nm = 380.0 + 5.0 * k;
    if (nm < h.begin || nm > h.end) return 0.0;
    return h.s[std::min((int)((nm - h.begin) * h.n / (h.end - h.begin)), (int)h.n - 1)];
}
inline double PowerHeuristic(double a, double b) { return a * a / (a * a + b * b); }

// SampledWavelengths::SampleEquidistant (SampledWavelengths.h:79-106): hero
// uniform in [lmin, lmax], companions a quarter range apart with wrap-around.
inline void Wavelengths(double u, double lmin, double lmax, double lam[4])
{
    const double range = lmax - lmin;
    lam[0] = lmin + u * range;
    for (int i = 1; i < 4; ++i) lam[i] = lmin + std::fmod(lam[0] - lmin + i * (range / 4.0), range);
}

// EvaluateRussianRoulette (PathTransportUtilities.h:86-110): returns true to
// terminate; `survival` is the probability to divide by (1 when not applied).
inline bool RussianRoulette(int depth, int minDepth, double threshold, double cur, double prev, double u,
                            double& survival)
{
    survival = 1.0;
    if (depth < minDepth) return false;
    const double prob = std::min(1.0, cur / std::max(prev, threshold));
    if (u >= prob) return true;
    if (prob > 0 && prob < 1) survival = prob;
    return false;
}

// amb: the index of the medium around the hit, the top of the path's
// index-of-refraction stack (PathTracingIntegrator.cpp:4315-4322), which the
// conductor Fresnel and its hemispherical average take as the incident index
// (GGXBRDF.cpp:430-434,476-481).
Ggx GgxAt(const Scene& S, int mat, double lam, double amb)
{
    Ggx g;
    g.amb = amb;
    g.alpha = std::max((double)S.mf[2 * mat], 1e-4);
    const int refl = S.mi[5 * mat + 1], eta = S.mi[5 * mat + 3], kap = S.mi[5 * mat + 4];
    g.spec = refl >= 0 ? Spec(S, refl, lam) : 1.0;
    g.eta = eta >= 0 ? Spec(S, eta, lam) : (double)S.mf[2 * mat + 1];
    g.k = kap >= 0 ? Spec(S, kap, lam) : 0.0;
    g.favg = FresnelAvg(amb, g.eta, g.k);
    return g;
}

// GGXBRDF::valueNM (r towards the viewer, v towards the light).
double GgxValue(const Ggx& g, V n, V gn, V r, V v)
{
    const double nr = Dot(n, r), nv = Dot(n, v);
    if (nr < kNearZero || nv < kNearZero) return 0.0;
    if (Dot(v, gn) <= 0 || Dot(r, gn) <= 0) return 0.0;
    const V h = Norm(v + r);
    const double G2 = 1.0 / (1.0 + Lambda(g.alpha, nv) + Lambda(g.alpha, nr));
    double f = 0.0;
    const double sf = GgxD(g.alpha, Dot(h, n)) * G2 / (4.0 * nv * nr);
    if (sf > 0) f = g.spec * ConductorF(Dot(r, h), g.amb, g.eta, g.k) * sf;
    const double eavg = LookupEavg(g.alpha);
    if (1.0 - eavg > 1e-10)
        f += Fms(g.spec * g.favg, eavg) * (1.0 - LookupEss(nr, g.alpha)) * (1.0 - LookupEss(nv, g.alpha)) / (kPi * (1.0 - eavg));
    return f;
}
double GgxPdf(const Ggx& g, V n, V gn, V r, V v)
{
    const double cv = Dot(v, n);
    if (cv <= 0 || Dot(v, gn) <= 0) return 0.0;
    const double ws = g.spec, wms = ws * (1.0 - LookupEss(Dot(r, n), g.alpha)), total = ws + wms;
    if (total < 1e-10) return cv * kInvPi;
    return (wms * MsPdf(cv, g.alpha, MsZ(g.alpha)) + ws * VndfPdf(r, v, n, g.alpha)) / total;
}

void EvalBsdf(const Scene& S, int mat, double lam, double amb, V ns, V gn, V r, V v, double& f, double& pdf)
{
    if (S.mi[5 * mat] == 1) {
        const V n = Dot(r, ns) < 0 ? -ns : ns;
        const Ggx g = GgxAt(S, mat, lam, amb);
        f = GgxValue(g, n, gn, r, v);
        pdf = GgxPdf(g, n, gn, r, v);
    } else {
        const double nr = Dot(ns, r), nv = Dot(ns, v);
        const bool same = (nr >= kNearZero && nv >= kNearZero) || (nr <= -kNearZero && nv <= -kNearZero);
        const bool gate = Dot(v, gn) > 0 && Dot(r, gn) > 0;
        f = (same && gate) ? Spec(S, S.mi[5 * mat + 1], lam) * kInvPi : 0.0;
        pdf = (same && gate) ? std::fabs(nv) * kInvPi : 0.0;
    }
}

double DielectricR(double cosI, double cosT, double ni, double nt)
{
    const double nn = ni * nt, cc = cosT * cosI, ni2 = ni * ni, nt2 = nt * nt;
    const double ci2 = cosI * cosI, ct2 = cosT * cosT, nit = ni2 - nt2, cit = ci2 - ct2;
    const double num = nit * nit * cc * cc + cit * cit * nn * nn;
    double den = cc * (ni2 + nt2) + nn * (ci2 + ct2);
    den *= den;
    if (den < 1e-6 && num < 1e-6) return 1.0;
    return std::min(1.0, num / den);
}

V OctDecode(unsigned q)
{
    const double u = (double)(float)((short)(q & 0xffffu) * (1.0f / 32767.0f));
    const double v = (double)(float)((short)(q >> 16) * (1.0f / 32767.0f));
    double x = u, y = v;
    const double z = 1.0 - std::fabs(u) - std::fabs(v);
    if (z < 0.0) {
        x = (1.0 - std::fabs(v)) * (u >= 0.0 ? 1.0 : -1.0);
        y = (1.0 - std::fabs(u)) * (v >= 0.0 ? 1.0 : -1.0);
    }
    return Norm(V{x, y, z});
}

// The reference's Moller-Trumbore barycentrics (alpha, beta) of a hit
// triangle (RayTriangleIntersection.cpp:36-60).
void Barycentrics(V o, V d, V a, V b, V c, double& al, double& be)
{
    const V ea = b - a, eb = c - a;
    const V pv = Cross(d, eb);
    const double det = Dot(ea, pv);
    const V tv = o - a;
    const V qv = Cross(tv, ea);
    al = Dot(tv, pv) / det;
    be = Dot(d, qv) / det;
}

// Hash key, or the pixel's Sobol seed, and the camera's numbers (dimensions
// 0-2: jitter x, y, hero wavelength).
inline uint32_t SampleKey(const Scene& S, uint32_t pixel, uint32_t sample)
{
    if (S.sampler != 0)
        return SobolPixelSeed(pixel % (uint32_t)S.width, pixel / (uint32_t)S.width, S.seed);
    return PathKey(S.seed, pixel, sample);
}
inline double CameraRand(const Scene& S, uint32_t key, uint32_t sample, uint32_t dim)
{
    return S.sampler != 0 ? SobolSample(sample, dim, key, S.sampler == 2) : Rand(key, dim);
}

void Sample(const Scene& S, uint32_t pixel, uint32_t sample, double xyz[3])
{
    const uint32_t key = SampleKey(S, pixel, sample);
    const int px = (int)(pixel % (uint32_t)S.width), py = (int)(pixel / (uint32_t)S.width);
    // Screen position, pixel centres on integer coordinates, rows downwards:
    // ptOnScreen = (x + u - 1/2, (height - y) + v - 1/2)
    // (PathTracingSpectralRasterizer.cpp:321-331, BoxPixelFilter.h:54-58), or
    // GaussianPixelFilter::warp about the pixel centre
    // (Sampling/GaussianPixelFilter.h:109-127); the pinhole maps it to the
    // direction W + (x - width/2) h ar / width (-U) + (height/2 - y_row) h / height V
    // (PinholeCamera.cpp:85-89,182-192,209-214).
    const double ox = CameraRand(S, key, sample, 0), oy = CameraRand(S, key, sample, 1);
    double fx = px + ox - 0.5, fy = py + 0.5 - oy;
    if (S.warpSigma > 0.0) {
        const double v = std::max(S.warpTrunc + (1.0 - S.warpTrunc) * ox, 1e-30);
        const double r = S.warpSigma * std::sqrt(-2.0 * std::log(v));
        const double th = 2.0 * kPi * oy;
        fx = px + r * std::cos(th);
        fy = py - r * std::sin(th);
    }
    const double sx = 2.0 * fx / S.width - 1.0, sy = 1.0 - 2.0 * fy / S.height;
    V d = Norm(S.fwd + S.right * sx + S.up * sy);
    V o = S.pos;
    // The hero of an equidistant bundle, or one wavelength, binned as the
    // reference's single-wavelength loop bins it
    // (PathTracingSpectralRasterizer.cpp:180-183); the companions of a
    // single-wavelength path start terminated.  The bin index is taken in
    // FP32 as the device takes it.
    double lam[4];
    const double uw = CameraRand(S, key, sample, 2);
    Wavelengths(uw, S.lmin, S.lmax, lam);
    if (S.single && S.numWl)
        lam[0] = S.lmin + std::min((int)((float)uw * (float)S.numWl), S.numWl - 1) * S.wlStep;
    unsigned term = S.single ? 0xeu : 0u;
    auto live = [&](int k) { return !((term >> k) & 1u); };
    double thr[4] = {1, 1, 1, 1}, L[4] = {0, 0, 0, 0};
    double bsdfPdf = 0.0;
    int bounces[3] = {0, 0, 0};
    // The index-of-refraction stack (Utilities/IORStack.h): the meshes the
    // path is inside, innermost last, over air; each entry's index is its
    // material's at the hero wavelength.
    std::vector<int> inside;
    auto iorOf = [&](int m) {
        const int mm = (int)S.meshes[4 * m + 2], sp = S.mi[5 * mm + 3];
        return sp >= 0 ? Spec(S, sp, lam[0]) : (double)S.mf[2 * mm + 1];
    };
    for (int depth = 0; depth < S.maxDepth; ++depth) {
        VertexRng rng{key, sample, depth, S.sampler, 0u};
        double mx = 0.0;
        bool bad = false;
        for (double v : thr) { if (!std::isfinite(v)) bad = true; mx = std::max(mx, std::fabs(v)); }
        if (bad || mx > 1e6) break;
        const double od[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        double t;
        const int prim = orc_closest_d(S.bvh, od, dd, &t);
        if (prim < 0) {
            if (S.envImg.rgb && (depth > 0 || S.envVisible)) {
                double c[3], sc, w = 1.0;
                S.envImg.Lookup(d, c, sc);
                if (bsdfPdf > 0) {
                    const double ep = S.envImg.Pdf(d);
                    if (ep > 0) w = PowerHeuristic(bsdfPdf, ep);
                }
                for (int k = 0; k < 4; ++k)
                    if (live(k)) L[k] += thr[k] * EnvImage::Spectrum(c, sc, lam[k]) * w;
            } else if (S.env >= 0 && (depth > 0 || S.envVisible)) {
                const double w = bsdfPdf > 0 ? PowerHeuristic(bsdfPdf, kInv4Pi) : 1.0;
                for (int k = 0; k < 4; ++k)
                    if (live(k)) L[k] += thr[k] * Spec(S, S.env, lam[k]) * w;
            }
            break;
        }
        const V p = o + d * t;
        const float* tv = S.tri9 + 9 * (size_t)prim;
        const V a = {tv[0], tv[1], tv[2]}, b = {tv[3], tv[4], tv[5]}, c = {tv[6], tv[7], tv[8]};
        const V nface = Norm(Cross(b - a, c - a));
        const int mesh = S.triMesh[prim];
        const int mat = (int)S.meshes[4 * mesh + 2];
        const bool ds = S.meshes[4 * mesh + 3] != 0;
        const int light = S.meshLight[mesh];
        const double amb = inside.empty() ? 1.0 : iorOf(inside.back());
        int stackOp = 0;   // 1: push this mesh; -1 - i: remove entry i
        // Shading normal: vertex normals interpolated at the hit, normalised
        // (TriangleMeshGeometryIndexedSpecializations.h:194-199, Object.cpp:543);
        // geometric normal: the face normal on the shading normal's side.
        V ns0 = nface;
        if (!S.octN.empty() && (S.octN[3 * prim] | S.octN[3 * prim + 1] | S.octN[3 * prim + 2])) {
            double al, be;
            Barycentrics(o, d, a, b, c, al, be);
            const V n0 = OctDecode(S.octN[3 * prim]), n1 = OctDecode(S.octN[3 * prim + 1]),
                    n2 = OctDecode(S.octN[3 * prim + 2]);
            ns0 = Norm(n0 + (n1 - n0) * al + (n2 - n0) * be);
        }
        V ng = Dot(nface, ns0) < 0 ? -nface : nface;
        V nsv = ns0;
        // Double-sided: both turned towards the ray (TriangleMeshGeometryIndexed.cpp:170-188).
        if (ds) {
            if (Dot(nsv, d) > 0) nsv = -nsv;
            if (Dot(ng, d) > 0) ng = -ng;
        }
        const V gnv = Dot(ng, d) < 0 ? ng : -ng;
        const int type = S.mi[5 * mat], refl = S.mi[5 * mat + 1], emit = S.mi[5 * mat + 2];
        if (emit >= 0 && Dot(-d, ng) > 0) {
            double w = 1.0;
            if (bsdfPdf > 0 && light >= 0) {
                const Light& lg = S.lights[light];
                const double cosL = std::fabs(Dot(d, ng));
                const double po[3] = {o.x, o.y, o.z};   // the previous vertex
                const double psel = S.lightBvh ? LightBvhPdf(S.lightNodes, lg.bvhPos, po) : lg.pdf;
                if (cosL > 0 && lg.area > 0) w = PowerHeuristic(bsdfPdf, psel * t * t / (lg.area * cosL));
            }
            for (int k = 0; k < 4; ++k)
                if (live(k)) L[k] += thr[k] * Spec(S, emit, lam[k]) * w;
        }
        double kray[4] = {0, 0, 0, 0};
        V nd;
        double npdf = 0.0;
        int btype = 0;   // continuation: 0 diffuse, 1 glossy, 2 transmission
        if (type == 2) {
            // Smooth dielectric (DielectricSPF.cpp:120-300) at the hero's
            // index; a constant index keeps the bundle together, a companion
            // whose index differs by more than 1e-8 ends with the others
            // (TerminateSecondary, PathTracingIntegrator.cpp:4658-4677).
            const int iorSpec = S.mi[5 * mat + 3];
            const double ior = iorSpec >= 0 ? Spec(S, iorSpec, lam[0]) : (double)S.mf[2 * mat + 1];
            if (iorSpec >= 0 && (term & 0xeu) != 0xeu)
                for (int k = 1; k < 4; ++k)
                    if (live(k) && std::fabs(Spec(S, iorSpec, lam[k]) - ior) > 1e-8) {
                        term |= 0xeu;
                        break;
                    }
            // Inside or outside from the path's index stack, not the facing
            // (DielectricSPF.cpp:406-418): inside, the ray leaves for the
            // medium under this mesh's entry (:177-183); outside, it comes
            // from the stack's top (:198-207).  w is ri.onb.w(), the shading
            // normal, turned towards the ray on a double-sided mesh.
            int pos = -1;
            for (int i = (int)inside.size() - 1; i >= 0; --i)
                if (inside[i] == mesh) { pos = i; break; }
            const bool fromInside = pos >= 0;
            double exitIor = 1.0;
            if (fromInside) {
                const int nIn = (int)inside.size();
                if (pos == nIn - 1) exitIor = nIn > 1 ? iorOf(inside[nIn - 2]) : 1.0;
                else exitIor = iorOf(inside[nIn - 1]);
            }
            const double n1 = fromInside ? ior : amb, n2 = fromInside ? exitIor : ior;
            const V w = nsv;
            const V nEff = fromInside ? -w : w;
            V geomN = Dot(ng, nEff) >= 0 ? ng : -ng;
            // Snell's law with the normal turned against the ray
            // (Optics.cpp:84-98); Fresnel on absolute cosines (:101-159).
            const V nf = Dot(w, d) > 0 ? -w : w;
            const double cosI = -Dot(d, nf), eta = n1 / n2;
            const double s2t = eta * eta * std::max(0.0, 1.0 - cosI * cosI);
            double R = 1.0;
            V tdir = {0, 0, 0};
            const bool snell = 1.0 - s2t >= kNearZero;
            if (snell) {
                const double cosT = std::sqrt(1.0 - s2t);
                tdir = Norm(d * eta + nf * (eta * cosI - cosT));
                R = DielectricR(cosI, cosT, n1, n2);
            }
            // ScatterNM's two numbers tilt the transmitted direction by the
            // material's Phong lobe (DielectricSPF.cpp:248-272; none at an
            // exponent of 0 or >= 1e6, mf[0] holding it for a dielectric).
            const double u1 = rng.next(16), u2 = rng.next(17);
            const double expo = S.mf[2 * mat];
            bool refr = snell;
            if (refr && expo > 0 && expo < 1e6) {
                const double al = std::acos(std::pow(u1, 1.0 / (expo + 1.0)));
                if (al > 0 && al < 0.5 * kPi) {
                    V tx, ty;
                    Frame(tdir, tx, ty);
                    const double ph = 2.0 * kPi * u2;
                    tdir = Norm(tdir * std::cos(al) + (tx * std::cos(ph) + ty * std::sin(ph)) * std::sin(al));
                }
            }
            // Transmission must cross to the far side of w's crossing;
            // reflection must stay above the geometric normal on that side,
            // mirrored about it under total internal reflection
            // (:221-243, :274-279).
            if (refr && !(Dot(tdir, nEff) < -kNearZero)) refr = false;
            V rdir = Norm(d - w * (2.0 * Dot(d, w)));
            bool refl = true;
            if (!(Dot(rdir, geomN) > 0)) {
                if (R >= 1.0) rdir = Norm(d - geomN * (2.0 * Dot(d, geomN)));
                else refl = false;
            }
            // RandomlySelect over (transmitted 1 - R, reflected R); the
            // transmitted ray carries the stack with this mesh pushed or
            // removed (PathTracingIntegrator.cpp:4814-4816).
            if (rng.next(18) < 1.0 - R) {
                if (!refr) break;
                nd = tdir;
                btype = 2;
                stackOp = fromInside ? -1 - pos : 1;
            } else {
                if (!refl) break;
                nd = rdir;
                btype = 1;
            }
            for (int k = 0; k < 4; ++k) kray[k] = live(k) ? 1.0 : 0.0;
        } else {
            const V ns = nsv, r = -d;
            const int nsamp = S.neePerLambda ? 4 : 1;
            for (int k = 0; k < nsamp; ++k) {
                if (S.neePerLambda && !live(k)) continue;
                if (!S.lights.empty()) {
                    const double ul = rng.next(4 * k);
                    int li = 0;
                    double psel;
                    if (S.lightBvh) {
                        const double pp[3] = {p.x, p.y, p.z};
                        li = SampleLightBvh(S.lightNodes, pp, ul, psel);
                    } else {
                        // AliasTable::Sample.
                        const int nl = (int)S.lights.size();
                        const double sc = ul * nl;
                        const int idx = std::min((int)sc, nl - 1);
                        li = (sc - idx < S.aliasProb[idx]) ? idx : S.aliasOf[idx];
                        psel = S.lights[li].pdf;
                    }
                    if (li >= 0 && S.lights[li].kind == 1 && psel > 0) {
                        // Point light (LightSampler.cpp:2097-2130): luminance of
                        // colour x power at every wavelength, cos / d^2, no MIS.
                        const Light& lg = S.lights[li];
                        V toL = lg.pos - p;
                        const double dist = std::sqrt(Dot(toL, toL));
                        toL = toL * (1.0 / dist);
                        const double cosS = Dot(toL, ns);
                        const double pd[3] = {p.x, p.y, p.z}, ld[3] = {toL.x, toL.y, toL.z};
                        if (cosS > 0 && !orc_any_d(S.bvh, pd, ld, dist - 0.001)) {
                            for (int j = 0; j < 4; ++j) {
                                if ((S.neePerLambda && j != k) || !live(j)) continue;
                                double f, pb;
                                EvalBsdf(S, mat, lam[j], amb, ns, gnv, r, toL, f, pb);
                                L[j] += thr[j] * lg.le * f * cosS / (dist * dist) / psel;
                            }
                        }
                    } else if (li >= 0 && li != light && psel > 0) {
                        const Light& lg = S.lights[li];
                        const double ux = rng.next(4 * k + 1), uy = rng.next(4 * k + 2), uz = rng.next(4 * k + 3);
                        // std::lower_bound over the areas CDF (TriangleMeshGeometryIndexed.cpp:207-217).
                        int ts = lg.first, hi = lg.first + lg.count - 1;
                        while (ts < hi) {
                            const int mid = (ts + hi) >> 1;
                            if (S.ltris[mid].cdf >= uz) hi = mid;
                            else ts = mid + 1;
                        }
                        const LTri& lt = S.ltris[ts];
                        const double sa = std::sqrt(1.0 - ux);
                        const V pl = lt.v0 + lt.e1 * (1.0 - sa) + lt.e2 * (sa * uy);
                        const V nl = Norm(Cross(lt.e1, lt.e2));
                        V toL = pl - p;
                        const double dist = std::sqrt(Dot(toL, toL));
                        toL = toL * (1.0 / dist);
                        const double cosS = Dot(toL, ns), cosL = Dot(-toL, nl);
                        const double pd[3] = {p.x, p.y, p.z}, ld[3] = {toL.x, toL.y, toL.z};
                        if (cosL > 0 && cosS > 0 && !orc_any_d(S.bvh, pd, ld, dist - 0.001)) {
                            const double geom = lg.area * cosL / (dist * dist);
                            const double plight = psel * dist * dist / (lg.area * cosL);
                            for (int j = 0; j < 4; ++j) {
                                if ((S.neePerLambda && j != k) || !live(j)) continue;
                                double f, pb;
                                EvalBsdf(S, mat, lam[j], amb, ns, gnv, r, toL, f, pb);
                                const double w = (pb > 0 ? PowerHeuristic(plight, pb) : 1.0) / psel;
                                L[j] += thr[j] * Spec(S, lg.emit, lam[j]) * cosS * geom * f * w;
                            }
                        }
                    } else if (!(li >= 0 && S.lights[li].kind == 1 && psel > 0)) {
                        // Nothing to sample, or the luminary being shaded: the
                        // reference still draws the point's three numbers
                        // (LightSampler.cpp:2064-2096).
                        rng.skip(3);
                    }
                }
                if (S.env >= 0 || S.envImg.rgb) {
                    // Environment NEE (LightSampler.cpp:2271-2359): the image's
                    // importance tables, or uniform directions for a uniform sky.
                    const double u1 = rng.next(20 + 2 * k), u2 = rng.next(21 + 2 * k);
                    V dir;
                    double epdf, ec[3] = {0, 0, 0}, esc = 0;
                    if (S.envImg.rgb) {
                        epdf = S.envImg.Sample(u1, u2, dir);
                        if (epdf > 0) S.envImg.Lookup(dir, ec, esc);
                    } else {
                        const double z = 1.0 - 2.0 * u1, rr = std::sqrt(std::max(0.0, 1.0 - z * z));
                        dir = {rr * std::cos(2.0 * kPi * u2), rr * std::sin(2.0 * kPi * u2), z};
                        epdf = kInv4Pi;
                    }
                    const double cosE = Dot(dir, ns);
                    const double pd[3] = {p.x, p.y, p.z}, ed[3] = {dir.x, dir.y, dir.z};
                    if (cosE > 0 && epdf > 0 && !orc_any_d(S.bvh, pd, ed, 1e300)) {
                        for (int j = 0; j < 4; ++j) {
                            if ((S.neePerLambda && j != k) || !live(j)) continue;
                            double f, pb;
                            EvalBsdf(S, mat, lam[j], amb, ns, gnv, r, dir, f, pb);
                            const double w = pb > 0 ? PowerHeuristic(epdf, pb) : 1.0;
                            const double le = S.envImg.rgb ? EnvImage::Spectrum(ec, esc, lam[j]) : Spec(S, S.env, lam[j]);
                            L[j] += thr[j] * le * f * cosE / epdf * w;
                        }
                    }
                }
            }
            const V w = Dot(d, ns) > kNearZero ? -ns : ns;
            const V gn = gnv;
            V tx, ty;
            Frame(w, tx, ty);
            const double ulobe = type == 1 ? rng.next(18) : 0.0;   // GGXSPF draws the lobe first
            const double u1 = rng.next(16), u2 = rng.next(17);
            if (type == 1) {
                const Ggx g0 = GgxAt(S, mat, lam[0], amb);
                const double cosR = Dot(r, w);
                const double ws = g0.spec, wms = ws * (1.0 - LookupEss(cosR, g0.alpha)), total = ws + wms;
                if (!(total > 1e-10)) break;
                const double pSpec = ws / total, pMS = wms / total;
                const double msz = MsZ(g0.alpha);
                double khero;
                if (ulobe < pSpec) {
                    btype = 1;
                    const V wl = {Dot(r, tx), Dot(r, ty), Dot(r, w)};
                    const V ml = VndfLocal(wl, g0.alpha, u1, u2);
                    const V mh = Norm(tx * ml.x + ty * ml.y + w * ml.z);
                    const double rm = Dot(r, mh);
                    if (!(rm > 0)) break;
                    nd = Norm(mh * (2.0 * rm) - r);
                    const double cosO = Dot(nd, w);
                    if (!(cosO > 0 && Dot(nd, gn) > 0)) break;
                    const double vpdf = VndfPdf(r, nd, w, g0.alpha);
                    if (!(vpdf > 1e-10)) break;
                    npdf = (wms * MsPdf(cosO, g0.alpha, msz) + ws * vpdf) / total;
                    const double G2 = 1.0 / (1.0 + Lambda(g0.alpha, cosR) + Lambda(g0.alpha, cosO));
                    const double G1 = 1.0 / (1.0 + Lambda(g0.alpha, cosR));
                    khero = g0.spec * ConductorF(rm, amb, g0.eta, g0.k) * G2 / (G1 * pSpec);
                } else {
                    // Multiple-scattering lobe: mu from (1 - E_ss(mu)) mu, uniform azimuth.
                    const double eavg = LookupEavg(g0.alpha);
                    if (!(pMS > 1e-10 && 1.0 - eavg > 1e-10)) break;
                    const double cost = MsSampleCos(g0.alpha, u1), sint = std::sqrt(std::max(0.0, 1.0 - cost * cost));
                    const double phi = 2.0 * kPi * u2;
                    nd = Norm(tx * (std::cos(phi) * sint) + ty * (std::sin(phi) * sint) + w * cost);
                    const double cosO = Dot(nd, w);
                    if (!(cosO > 0 && Dot(nd, gn) > 0)) break;
                    const double mpdf = MsPdf(cosO, g0.alpha, msz);
                    npdf = (wms * mpdf + ws * VndfPdf(r, nd, w, g0.alpha)) / total;
                    const double fms = Fms(g0.spec * g0.favg, eavg) * (1.0 - LookupEss(cosO, g0.alpha)) *
                                       (1.0 - LookupEss(cosR, g0.alpha)) / (kPi * (1.0 - eavg));
                    if (!(mpdf > 1e-14)) break;
                    khero = fms * cosO / (mpdf * pMS);
                }
                if (!(npdf > 0)) break;
                kray[0] = live(0) ? khero : 0.0;
                const double cosV = std::fabs(Dot(nd, ns));
                for (int k = 1; k < 4; ++k)
                    kray[k] = live(k) ? GgxValue(GgxAt(S, mat, lam[k], amb), w, gnv, r, nd) * cosV / npdf : 0.0;
            } else {
                const double phi = 2.0 * kPi * u1, sint = std::sqrt(u2), cost = std::sqrt(1.0 - u2);
                nd = Norm(tx * (std::cos(phi) * sint) + ty * (std::sin(phi) * sint) + w * cost);
                npdf = std::fabs(Dot(nd, w)) * kInvPi;
                if (!(Dot(nd, gn) > 0)) break;
                for (int k = 0; k < 4; ++k) kray[k] = live(k) ? Spec(S, refl, lam[k]) : 0.0;
            }
        }
        if (type != 2) rng.skip(1);   // the integrator's choice among the scattered rays (a dielectric's is its Fresnel choice)
        double prevMax = 0, currMax = 0;
        for (int k = 0; k < 4; ++k) {
            if (!live(k)) continue;
            prevMax = std::max(prevMax, std::fabs(thr[k]));
            currMax = std::max(currMax, std::fabs(thr[k] * kray[k]));
        }
        if (currMax <= kNearZero) break;
        double survival;
        if (depth >= S.rrMinDepth &&
            RussianRoulette(depth, S.rrMinDepth, S.rrThreshold, currMax, prevMax, rng.next(19), survival))
            break;
        if (depth < S.rrMinDepth) survival = 1.0;
        if (survival != 1.0)
            for (double& k : kray) k /= survival;
        // Per-type bounce limits, after Russian roulette
        // (PropagateBounceLimits, PathTransportUtilities.h:170-221).
        if (++bounces[btype] > S.maxBounce[btype]) break;
        if (depth + 1 >= S.maxDepth) break;
        for (int k = 0; k < 4; ++k) thr[k] *= kray[k];
        if (stackOp > 0) inside.push_back(mesh);
        else if (stackOp < 0) inside.erase(inside.begin() + (-1 - stackOp));
        bsdfPdf = npdf;
        o = p + nd * 1e-8;   // Ray::Advance(1e-8), PathTracingIntegrator.cpp:4812
        d = nd;
    }
    xyz[0] = xyz[1] = xyz[2] = 0.0;
    int active = 0;
    for (int k = 0; k < 4; ++k) {
        int i, j;
        double wgt;
        if (!live(k) || !Interp(lam[k], i, j, wgt)) continue;
        for (int c = 0; c < 3; ++c) {
            const double* tab = S.cie + 81 * c;
            xyz[c] += (tab[i] + wgt * (tab[j] - tab[i])) * L[k];
        }
        ++active;
    }
    if (active > 0)
        for (int c = 0; c < 3; ++c) xyz[c] *= S.ynorm / active;
}

}  // namespace

namespace {

// Adaptive sampling settings (Utilities/AdaptiveSamplingConfig.h): off when
// max_spp is 0.
struct Adaptive {
    int max_spp = 0;
    int batch = 0;
    double threshold = 0.01;
};

// The per-pixel sample loop of PathTracingSpectralRasterizer::IntegratePixel
// (Rendering/PathTracingSpectralRasterizer.cpp:256-410).  Without adaptive
// sampling: spp samples from sample_begin.  With it: batches of A.batch
// samples from sample 0, a Welford running mean / M2 of each sample's
// luminance (XYZ.Y), and after every batch, once 32 samples are in, the
// convergence test -- standard error / |mean| below threshold * (1 - 4 / N),
// or M2 < 1e-12 after 64 samples for a black pixel -- until it passes or
// A.max_spp samples are taken.  emit(path, xyz) sees every path (a pixel
// sample is S.spectral paths, numbered sample * S.spectral + j); the return
// value is the number of pixel samples taken.
template <class F>
int PixelSamples(const Scene& S, uint32_t pixel, int sample_begin, int spp, const Adaptive& A, F&& emit)
{
    double v[3];
    if (A.max_spp <= 0) {
        for (int s = 0; s < spp; ++s)
            for (int j = 0; j < S.spectral; ++j) {
                const uint32_t path = (uint32_t)((sample_begin + s) * S.spectral + j);
                Sample(S, pixel, path, v);
                emit(path, v);
            }
        return spp;
    }
    double mean = 0.0, m2 = 0.0;
    unsigned n = 0;
    int idx = 0;
    bool converged = false;
    while (idx < A.max_spp && !converged) {
        const int end = std::min(idx + A.batch, A.max_spp);
        for (; idx < end; ++idx) {
            Sample(S, pixel, (uint32_t)idx, v);
            emit((uint32_t)idx, v);
            ++n;
            const double d = v[1] - mean;
            mean += d / (double)n;
            m2 += d * (v[1] - mean);
        }
        if (n >= 32) {
            const double se = std::sqrt(m2 / (double)(n - 1) / (double)n), ma = std::fabs(mean);
            if (ma > 1e-12) {
                if (se / ma < A.threshold * (1.0 - 4.0 / (double)n)) converged = true;
            } else if (m2 < 1e-12 && n >= 64) {
                converged = true;
            }
        }
    }
    return idx;
}

}  // namespace

// ---- colour resolve and 8-bit output ----------------------------------------

namespace {

struct Chroma {
    double x, y;
};

// Rec.709 primaries and D65 white in CIE xy (Utilities/Color/ColorUtils.cpp:135-138).
const Chroma kRed709 = {0.640, 0.330}, kGreen709 = {0.300, 0.600}, kBlue709 = {0.150, 0.060},
             kWhite709 = {0.3127, 0.3290};

// LineIntersection2D (ColorUtils.cpp:145-177): the line a0-a1 against b0-b1,
// refused when |denominator| < 1e-12.
bool LinesMeet(Chroma a0, Chroma a1, Chroma b0, Chroma b1, Chroma& at)
{
    const double den = (b1.y - b0.y) * (a1.x - a0.x) - (b1.x - b0.x) * (a1.y - a0.y);
    if (den > -1e-12 && den < 1e-12) return false;
    const double ua = ((b1.x - b0.x) * (a0.y - b0.y) - (b1.y - b0.y) * (a0.x - b0.x)) / den;
    at.x = a0.x + ua * (a1.x - a0.x);
    at.y = a0.y + ua * (a1.y - a0.y);
    return true;
}

// IsPointOnLineSegment (ColorUtils.cpp:204-211): the parameter along x alone.
bool OnSegment(Chroma s0, Chroma s1, Chroma p)
{
    const double v = (p.x - s0.x) / (s1.x - s0.x);
    return v >= 1e-12 && v <= 1.0 - 1e-12;
}

// ClipAgainstGamutEdge (ColorUtils.cpp:213-229).
bool GamutEdge(Chroma c, Chroma a, Chroma b, Chroma& at)
{
    if (!LinesMeet(kWhite709, c, a, b, at)) return false;
    if (!OnSegment(a, b, at)) return false;
    if (OnSegment(kWhite709, at, c)) {
        at = c;
        return true;
    }
    return OnSegment(kWhite709, c, at);
}

double ToneCurve(int tone, double x)
{
    // DisplayTransforms (Rendering/DisplayTransform.h:80-222).
    const double s = (std::isfinite(x) && x > 0.0) ? x : 0.0;
    auto unit = [](double y) { return std::min(std::max(y, 0.0), 1.0); };
    auto hable = [](double v) {
        return ((v * (0.15 * v + 0.10 * 0.50) + 0.20 * 0.02) / (v * (0.15 * v + 0.50) + 0.20 * 0.30)) - 0.02 / 0.30;
    };
    switch (tone) {
    case 1: return s / (1.0 + s);
    case 2: return unit(s * (2.51 * s + 0.03) / (s * (2.43 * s + 0.59) + 0.14));
    case 3: return unit(0.5 + 0.5 * std::tanh(1.0 * (std::log10(s + 1e-10) - 0.0)));
    case 4: return unit(hable(s * 2.0) / hable(11.2));
    default: return s;
    }
}

}  // namespace

/* ColorUtils::XYZtoRec709RGB (Utilities/Color/Color.cpp:214-228): gamut
 * move of the chromaticity (MoveXYZIntoRec709RGBGamut, ColorUtils.cpp:351-363:
 * edges red-green, red-blue, blue-green in that order; xyY round trip,
 * Color.cpp:169-193), then the XYZ -> Rec.709 matrix (Color.cpp:22-25). */
extern "C" void orc_pt_xyz_to_rec709(const double* xyz, double* rgb)
{
    double X = xyz[0], Y = xyz[1], Z = xyz[2];
    const double inv = 1.0 / (X + Y + Z);
    const Chroma c = {X * inv, Y * inv};
    Chroma at;
    if (GamutEdge(c, kRed709, kGreen709, at) || GamutEdge(c, kRed709, kBlue709, at) ||
        GamutEdge(c, kBlue709, kGreen709, at)) {
        const double k = 1.0 / at.y * Y;
        X = k * at.x;
        Z = k * (1.0 - at.x - at.y);
    }
    rgb[0] = 3.240479 * X + -1.537150 * Y + -0.498535 * Z;
    rgb[1] = -0.969256 * X + 1.875992 * Y + 0.041556 * Z;
    rgb[2] = 0.055648 * X + -0.204043 * Y + 1.057311 * Z;
}

/* One pixel of an 8-bit output: exposure 2^ev and tone curve
 * (DisplayTransformWriter::WriteColor, Rendering/DisplayTransformWriter.cpp:45-62),
 * sRGB transfer (ColorUtils::SRGBTransferFunction, ColorUtils.cpp:21-32),
 * clamp to [0, 1], x 255 truncated (Color_Template.h:115-134). */
extern "C" void orc_pt_display(const double* rgb, double exposure_ev, int tone, unsigned char* out3)
{
    const double mul = std::pow(2.0, exposure_ev);
    for (int k = 0; k < 3; ++k) {
        const double x = ToneCurve(tone, rgb[k] * mul);
        double v;
        if (x == 0.0) v = 0.0;
        else if (x <= 0.003040247678) v = 12.92 * x;
        else v = 1.055 * std::pow(x, 1.0 / 2.4) - 0.055;
        if (v > 1.0) v = 1.0;
        if (v < 0.0) v = 0.0;
        out3[k] = (unsigned char)(v * 255.0);
    }
}

/* The light BVH on its own, for the comparison with the reference's: n
 * point lights (positions 3n, powers n; boxes widened by 1e-12 as
 * EnsureBoxHasVolume does), m queries (points 3m, random numbers m): picked
 * light and selection probability per query, and the probability of every
 * light from every query point (m x n). */
extern "C" void orc_pt_light_bvh(int n, const double* pos, const double* power, int m, const double* pts,
                                 const double* xi, int* picked, double* pdf, double* pdf_all)
{
    std::vector<LightPrimD> prims(n);
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) {
            prims[i].lo[k] = pos[3 * i + k] - 1e-12;
            prims[i].hi[k] = pos[3 * i + k] + 1e-12;
            prims[i].c[k] = 0.5 * (prims[i].lo[k] + prims[i].hi[k]);
        }
        prims[i].power = power[i];
        prims[i].light = i;
    }
    std::vector<LightNode> nodes;
    std::vector<int> posOf(n, 0);
    int at = 0;
    BuildLightBvh(prims, 0, n, at, nodes, posOf);
    for (int q = 0; q < m; ++q) {
        picked[q] = SampleLightBvh(nodes, pts + 3 * q, xi[q], pdf[q]);
        for (int i = 0; i < n; ++i) pdf_all[(size_t)q * n + i] = LightBvhPdf(nodes, posOf[i], pts + 3 * q);
    }
}

/* GaussianPixelFilter::EvaluateFilter (Sampling/GaussianPixelFilter.h:67-78):
 * exp(-r^2 / (2 sigma^2)) / (2 pi sigma^2) inside the size x size box centred
 * on the pixel centre, 0 outside it. */
extern "C" double orc_pt_gaussian_weight(double size, double sigma, double dx, double dy)
{
    const double h = 0.5 * size;
    if (std::fabs(dx) > h || std::fabs(dy) > h) return 0.0;
    const double two_s2 = 2.0 * sigma * sigma;
    return 1.0 / (kPi * two_s2) * std::exp(-(dx * dx + dy * dy) / two_s2);
}

extern "C" int orc_pt_render(const float* tri9, int64_t n_tri, const int64_t* meshes, int32_t n_mesh,
                             const float* spectra, int32_t n_spec, const int32_t* mats_i, const float* mats_f,
                             int32_t n_mat, const int32_t* envi, const double* cam, const double* setd,
                             const int32_t* seti, int32_t spp, int32_t sample_begin, int32_t x0, int32_t y0,
                             int32_t x1, int32_t y1, int32_t threads, double* xyz, const double* cie,
                             int32_t* counts, int32_t n_point, const double* points, const float* nrm9,
                             const OrcEnvImage* env_image)
{
    (void)n_spec;
    GetTables();
    Scene S;
    if (env_image && env_image->rgb) {
        S.envImg.rgb = env_image->rgb;
        S.envImg.w = env_image->width;
        S.envImg.h = env_image->height;
        S.envImg.scale = env_image->scale;
        S.envImg.table = env_image->uplift;
        S.envImg.Rotation(env_image->orient_rad);
        S.envImg.Build();
    }
    S.tri9 = tri9;
    S.nrm9 = nrm9;
    if (nrm9) {
        // Encode as the device does: unit length in FP32, then OctEncode; a
        // triangle without normals (all zero) stays flat.
        S.octN.assign(3 * (size_t)n_tri, 0u);
        for (int64_t t = 0; t < n_tri; ++t) {
            const float* q = nrm9 + 9 * t;
            bool any = false;
            for (int k = 0; k < 9; ++k) any |= q[k] != 0.0f;
            if (!any) continue;
            for (int j = 0; j < 3; ++j) {
                const float* n = q + 3 * j;
                const float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                S.octN[3 * t + j] = OctEncode(n[0] / l, n[1] / l, n[2] / l);
            }
        }
    }
    S.meshes = meshes;
    S.spectra = spectra;
    S.mi = mats_i;
    S.mf = mats_f;
    S.cie = cie;
    S.env = envi[0];
    S.envVisible = envi[1];
    S.lmin = setd[0];
    S.lmax = setd[1];
    S.rrThreshold = setd[2];
    S.width = seti[0];
    S.height = seti[1];
    S.maxDepth = seti[2];
    S.rrMinDepth = seti[3];
    S.neePerLambda = seti[4];
    S.seed = (uint32_t)seti[5];
    S.sampler = seti[9];
    if (seti[10])
        for (int k = 0; k < 3; ++k) S.maxBounce[k] = std::min(seti[11 + k], 255);
    S.single = seti[14] == 1;
    S.numWl = seti[15] > 0 && seti[15] < 10000 ? seti[15] : 0;
    S.spectral = std::max(1, (int)seti[16]);
    {
        const double lo = std::max(S.lmin, 380.0), hi = std::min(S.lmax, 780.0);
        const int f = (int)((lo - 380.0) / 5.0), l = (int)((hi - 380.0) / 5.0);
        double ky = 0.0;
        for (int i = f; i < l; ++i) ky += 0.5 * (cie[81 + i] + cie[81 + i + 1]) * 5.0;
        S.ynorm = ky > 0 ? (S.lmax - S.lmin) / ky : 0.0;
        S.wlStep = S.numWl ? (float)((S.lmax - S.lmin) / S.numWl) : 0.0;
    }
    const V pos = {cam[0], cam[1], cam[2]}, look = {cam[3], cam[4], cam[5]}, upv = {cam[6], cam[7], cam[8]};
    const V f = Norm(look - pos);
    const V r = Norm(Cross(f, upv));
    const V u = Cross(r, f);
    const double th = std::tan(0.5 * cam[9] * kPi / 180.0);
    const double aspect = (double)S.width / S.height;
    S.pos = pos;
    S.fwd = f;
    S.right = r * (th * aspect);
    S.up = u * th;
    S.triMesh.assign((size_t)n_tri, 0);
    S.meshLight.assign((size_t)n_mesh, -1);
    std::vector<double> weight;
    std::vector<LightPrimD> lightPrims;
    for (int m = 0; m < n_mesh; ++m) {
        const int64_t first = meshes[4 * m], count = meshes[4 * m + 1];
        for (int64_t t = first; t < first + count; ++t) S.triMesh[t] = m;
        const int mat = (int)meshes[4 * m + 2];
        if (mat < 0 || mat >= n_mat) return 1;
        const int emit = mats_i[5 * mat + 2];
        if (emit < 0 || count <= 0) continue;
        Light lg;
        lg.first = (int)S.ltris.size();
        lg.count = (int)count;
        lg.emit = emit;
        double area = 0.0;
        std::vector<double> cum;
        for (int64_t t = first; t < first + count; ++t) {
            const float* v = tri9 + 9 * t;
            LTri lt;
            lt.v0 = {v[0], v[1], v[2]};
            lt.e1 = {(double)(v[3] - v[0]), (double)(v[4] - v[1]), (double)(v[5] - v[2])};
            lt.e2 = {(double)(v[6] - v[0]), (double)(v[7] - v[1]), (double)(v[8] - v[2])};
            const V cr = Cross(lt.e1, lt.e2);
            area += 0.5 * std::sqrt(Dot(cr, cr));
            cum.push_back(area);
            S.ltris.push_back(lt);
        }
        if (!(area > 0)) { S.ltris.resize(lg.first); continue; }
        for (size_t k = 0; k < cum.size(); ++k) S.ltris[lg.first + k].cdf = cum[k] / area;
        S.ltris[lg.first + cum.size() - 1].cdf = 1.0;
        lg.area = area;
        double mean = 0.0;
        for (int k = 0; k < 81; ++k) mean += GridValue(spectra, emit, k);
        mean /= 81.0;
        weight.push_back(area * std::max(mean, 1e-12));
        LightPrimD q;
        for (int k = 0; k < 3; ++k) { q.lo[k] = INFINITY; q.hi[k] = -INFINITY; }
        for (int64_t t = first; t < first + count; ++t)
            for (int j = 0; j < 9; ++j) {
                q.lo[j % 3] = std::min(q.lo[j % 3], (double)tri9[9 * t + j]);
                q.hi[j % 3] = std::max(q.hi[j % 3], (double)tri9[9 * t + j]);
            }
        for (int k = 0; k < 3; ++k) {
            if (q.lo[k] == q.hi[k]) { q.lo[k] -= 1e-12; q.hi[k] += 1e-12; }   // EnsureBoxHasVolume
            q.c[k] = 0.5 * (q.lo[k] + q.hi[k]);
        }
        q.power = weight.back();
        q.light = (int)S.lights.size();
        lightPrims.push_back(q);
        S.meshLight[m] = (int)S.lights.size();
        S.lights.push_back(lg);
    }
    // Point lights (Lights/PointLight.h:49-57; LightSampler.cpp:655-668 weighs
    // every light by its radiant exitance: max(colour x power) x 4 pi here
    // against area x pi x mean radiance for a luminary, so with the common pi
    // dropped, max(colour x power) x 4).
    for (int i = 0; i < n_point; ++i) {
        const double* q7 = points + 7 * i;
        // Lights of zero exitance are dropped (LightSampler::Prepare).
        if (!(std::max({(double)(float)q7[3], (double)(float)q7[4], (double)(float)q7[5]}) * (double)(float)q7[6] > 0))
            continue;
        Light lg;
        lg.first = lg.count = 0;
        lg.emit = -1;
        lg.area = 0.0;
        lg.kind = 1;
        lg.pos = {(double)(float)q7[0], (double)(float)q7[1], (double)(float)q7[2]};
        lg.le = (double)(float)(0.2126 * (float)q7[3] * (float)q7[6] + 0.7152 * (float)q7[4] * (float)q7[6] +
                                0.0722 * (float)q7[5] * (float)q7[6]);
        weight.push_back(std::max({(double)(float)q7[3], (double)(float)q7[4], (double)(float)q7[5]}) *
                         (double)(float)q7[6] * 4.0);
        LightPrimD q;
        for (int k = 0; k < 3; ++k) {
            q.lo[k] = (double)(float)q7[k] - 1e-12;
            q.hi[k] = (double)(float)q7[k] + 1e-12;
            q.c[k] = 0.5 * (q.lo[k] + q.hi[k]);
        }
        q.power = weight.back();
        q.light = (int)S.lights.size();
        lightPrims.push_back(q);
        S.lights.push_back(lg);
    }
    double wsum = 0.0;
    for (double w : weight) wsum += w;
    for (size_t i = 0; i < S.lights.size(); ++i) S.lights[i].pdf = weight[i] / wsum;
    {
        // Vose's alias table (Utilities/AliasTable.h:34-101), the stack order
        // of the reference; thresholds rounded to FP32 as the device keeps them.
        const size_t n = weight.size();
        std::vector<double> scaled(n);
        S.aliasProb.assign(n, 1.0);
        S.aliasOf.resize(n);
        std::vector<int> small, large;
        for (size_t i = 0; i < n; ++i) {
            scaled[i] = weight[i] / wsum * (double)n;
            S.aliasOf[i] = (int)i;
            (scaled[i] < 1.0 ? small : large).push_back((int)i);
        }
        while (!small.empty() && !large.empty()) {
            const int sm = small.back(), lg = large.back();
            small.pop_back();
            large.pop_back();
            S.aliasProb[sm] = scaled[sm];
            S.aliasOf[sm] = lg;
            scaled[lg] = (scaled[lg] + scaled[sm]) - 1.0;
            (scaled[lg] < 1.0 ? small : large).push_back(lg);
        }
        for (double& x : S.aliasProb) x = (double)(float)x;
    }
    if (seti[8] == 0 && S.lights.size() > 1) {
        std::vector<int> posOf(S.lights.size(), 0);
        int pos = 0;
        BuildLightBvh(lightPrims, 0, (int)lightPrims.size(), pos, S.lightNodes, posOf);
        for (size_t i = 0; i < S.lights.size(); ++i) S.lights[i].bvhPos = posOf[i];
        S.lightBvh = true;
    }
    S.bvh = orc_bvh_build(tri9, n_tri);
    const int cw = x1 - x0, ch = y1 - y0;
    Adaptive A;
    if (seti[7] > 0) {
        A.max_spp = seti[7];
        A.batch = spp;
        A.threshold = setd[5];
        if (sample_begin != 0 || spp <= 0) { orc_bvh_destroy(S.bvh); return 1; }
    }
    if (seti[6] == 1 && 0.5 * setd[3] <= 0.501) {
        // Too narrow for the filtered film (PixelBasedRasterizerHelper.cpp:143-149).
        const double k = 0.5 * setd[3] / setd[4];
        S.warpSigma = setd[4];
        S.warpTrunc = std::exp(-0.5 * k * k);
    } else if (seti[6] == 1) {
        // GaussianPixelFilter + FilteredFilm (Rendering/FilteredFilm.cpp:42-132):
        // every sample of the pixels within the support of the crop is
        // splatted at its screen position (uniform in its pixel, pixel centres
        // on integer coordinates); a crop pixel resolves to sum(w XYZ) / sum(w).
        const double size = setd[3], hw = 0.5 * setd[3], sigma = setd[4];
        const int m = (int)std::ceil(hw) + 1;
        const int ex0 = std::max(0, x0 - m), ex1 = std::min(S.width, x1 + m);
        const int ey0 = std::max(0, y0 - m), ey1 = std::min(S.height, y1 + m);
        const int nt = std::max(1, threads);
        std::vector<std::vector<double>> films(nt, std::vector<double>(4 * (size_t)cw * ch, 0.0));
        std::atomic<int> row(ey0);
        auto fwork = [&](int tid) {
            std::vector<double>& film = films[tid];
            for (int py; (py = row.fetch_add(1)) < ey1;) {
                for (int px = ex0; px < ex1; ++px) {
                    const uint32_t pixel = (uint32_t)(py * S.width + px);
                    auto splat = [&](uint32_t sample, const double* v) {
                        const uint32_t key = SampleKey(S, pixel, sample);
                        const double sx = px + CameraRand(S, key, sample, 0) - 0.5,
                                     sy = py + 0.5 - CameraRand(S, key, sample, 1);
                        const int qx0 = std::max(x0, (int)std::floor(sx - hw));
                        const int qx1 = std::min(x1 - 1, (int)std::floor(sx + hw));
                        const int qy0 = std::max(y0, (int)std::floor(sy - hw));
                        const int qy1 = std::min(y1 - 1, (int)std::floor(sy + hw));
                        for (int qy = qy0; qy <= qy1; ++qy)
                            for (int qx = qx0; qx <= qx1; ++qx) {
                                const double w = orc_pt_gaussian_weight(size, sigma, sx - qx, sy - qy);
                                if (w == 0.0) continue;
                                double* f = &film[4 * ((size_t)(qy - y0) * cw + (qx - x0))];
                                for (int c = 0; c < 3; ++c) f[c] += w * v[c];
                                f[3] += w;
                            }
                    };
                    const int n = PixelSamples(S, pixel, sample_begin, spp, A, splat);
                    if (counts && px >= x0 && px < x1 && py >= y0 && py < y1)
                        counts[(size_t)(py - y0) * cw + (px - x0)] = n;
                }
            }
        };
        std::vector<std::thread> fpool;
        for (int t = 0; t < nt; ++t) fpool.emplace_back(fwork, t);
        for (auto& t : fpool) t.join();
        for (size_t p = 0; p < (size_t)cw * ch; ++p) {
            double a[4] = {0, 0, 0, 0};
            for (const auto& film : films)
                for (int c = 0; c < 4; ++c) a[c] += film[4 * p + c];
            for (int c = 0; c < 3; ++c) xyz[3 * p + c] = std::fabs(a[3]) > 1e-10 ? a[c] / a[3] : 0.0;
        }
        orc_bvh_destroy(S.bvh);
        return 0;
    }
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            const int row = next.fetch_add(1);
            if (row >= ch) break;
            for (int x = 0; x < cw; ++x) {
                const uint32_t pixel = (uint32_t)((y0 + row) * S.width + (x0 + x));
                double acc[3] = {0, 0, 0};
                const double inv = 1.0 / S.spectral;
                const int n = PixelSamples(S, pixel, sample_begin, spp, A, [&](uint32_t, const double* v) {
                    for (int c = 0; c < 3; ++c) acc[c] += v[c] * inv;
                });
                for (int c = 0; c < 3; ++c) xyz[3 * ((size_t)row * cw + x) + c] = acc[c] / n;
                if (counts) counts[(size_t)row * cw + x] = n;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    orc_bvh_destroy(S.bvh);
    return 0;
}

// ---- building blocks, exported for the component checks against the
// reference's own code (tests only) ------------------------------------------

extern "C" {

void orc_pt_sample_wavelengths(double u, double lmin, double lmax, double* lam4) { Wavelengths(u, lmin, lmax, lam4); }

int orc_pt_xyz_from_nm(double nm, const double* cie, double* xyz3)
{
    int i, j;
    double w;
    xyz3[0] = xyz3[1] = xyz3[2] = 0.0;
    if (!Interp(nm, i, j, w)) return 0;
    for (int c = 0; c < 3; ++c) xyz3[c] = cie[81 * c + i] + w * (cie[81 * c + j] - cie[81 * c + i]);
    return 1;
}

double orc_pt_ggx_d(double alpha, double cosH) { return GgxD(alpha, cosH); }
double orc_pt_ggx_lambda(double alpha, double cosT) { return Lambda(alpha, cosT); }
double orc_pt_ggx_g2(double alpha, double ci, double co) { return 1.0 / (1.0 + Lambda(alpha, ci) + Lambda(alpha, co)); }

// Visible-normal sample in the frame (t, b, n), as the path sampler draws it.
void orc_pt_vndf_sample(const double* wi, const double* t, const double* b, const double* n, double alpha, double u1,
                        double u2, double* m)
{
    const V r = {wi[0], wi[1], wi[2]}, tx = {t[0], t[1], t[2]}, ty = {b[0], b[1], b[2]}, w = {n[0], n[1], n[2]};
    const V wl = {Dot(r, tx), Dot(r, ty), Dot(r, w)};
    const V ml = VndfLocal(wl, alpha, u1, u2);
    const V mh = Norm(tx * ml.x + ty * ml.y + w * ml.z);
    m[0] = mh.x; m[1] = mh.y; m[2] = mh.z;
}

double orc_pt_vndf_pdf(const double* wi, const double* wo, const double* n, double alpha)
{
    return VndfPdf({wi[0], wi[1], wi[2]}, {wo[0], wo[1], wo[2]}, {n[0], n[1], n[2]}, alpha);
}

double orc_pt_conductor_f(double cosI, double ni, double nt, double k) { return ConductorF(cosI, ni, nt, k); }
double orc_pt_dielectric_r(double cosI, double cosT, double ni, double nt) { return DielectricR(cosI, cosT, ni, nt); }
double orc_pt_lookup_ess(double c, double alpha) { return LookupEss(c, alpha); }
double orc_pt_lookup_eavg(double alpha) { return LookupEavg(alpha); }
double orc_pt_ms_z(double alpha) { return MsZ(alpha); }
double orc_pt_ms_pdf(double c, double alpha, double z) { return MsPdf(c, alpha, z); }
double orc_pt_ms_sample_cos(double alpha, double u) { return MsSampleCos(alpha, u); }
double orc_pt_fresnel_avg(double ni, double nt, double k) { return FresnelAvg(ni, nt, k); }
double orc_pt_fms(double favg, double eavg) { return Fms(favg, eavg); }
double orc_pt_power_heuristic(double a, double b) { return PowerHeuristic(a, b); }

// The device's Sobol sampler: out[i] = the 32-bit scrambled value of sample
// index[i], dimension dim[i], seed seed[i]; hc[i] = HashCombine(a[i], b[i]).
void orc_pt_sobol(const uint32_t* index, const uint32_t* dim, const uint32_t* seed, int64_t n, uint32_t* out)
{
    for (int64_t i = 0; i < n; ++i) out[i] = SobolBits(index[i], dim[i], seed[i]);
}
void orc_pt_hash_combine(const uint32_t* a, const uint32_t* b, int64_t n, uint32_t* out)
{
    for (int64_t i = 0; i < n; ++i) out[i] = HashCombine(a[i], b[i]);
}

int orc_pt_russian_roulette(int depth, int min_depth, double threshold, double cur, double prev, double u,
                            double* survival)
{
    return RussianRoulette(depth, min_depth, threshold, cur, prev, u, *survival) ? 1 : 0;
}

// Read the energy tables (E_ss 32 x 32 row-major by alpha, E_avg 32).
void orc_pt_tables(double* ess, double* eavg)
{
    const Tables& T = GetTables();
    for (int a = 0; a < 32; ++a) {
        for (int c = 0; c < 32; ++c) ess[32 * a + c] = T.ess[a][c];
        eavg[a] = T.eavg[a];
    }
}

// Replace the energy tables (to check the lookups and the sampler on the
// reference's own table values).  Not thread-safe: call with no render running.
void orc_pt_set_tables(const double* ess, const double* eavg)
{
    Tables& T = MutableTables();
    for (int a = 0; a < 32; ++a) {
        for (int c = 0; c < 32; ++c) T.ess[a][c] = ess[32 * a + c];
        T.eavg[a] = eavg[a];
    }
    ComputeMsZ(T);
}

}  // extern "C"
