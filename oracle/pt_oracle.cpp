// pt_oracle.cpp -- TEST INFRASTRUCTURE ONLY (oracle port).
//
// Double-precision, one-sample-at-a-time restatement of the reference's
// hero-wavelength spectral path tracer for the scenes of this project
// (triangle meshes, Lambertian surfaces, Lambertian area emitters, uniform
// sky):
//   * per-pixel sample loop, box pixel filter   PathTracingSpectralRasterizer.cpp:206-479
//   * 4 equidistant wavelengths, XYZ, (b-a)/k_y  PathTracingSpectralRasterizer.cpp:121-198,
//                                                SampledWavelengths.h:79-106,
//                                                ColorUtils.cpp:270-348
//   * bounce loop                               PathTracingIntegrator.cpp:4094-4817
//       runaway guard :4099-4110, emission + MIS :4424-4518, NEE per
//       wavelength :4523-4550, BSDF sample + companions :4597-4719,
//       Russian roulette :4738-4769, update + Advance(1e-8) :4791-4816
//   * area-light NEE                            LightSampler.cpp:2083-2271
//   * cosine sampling, Lambertian value/pdf     LambertianSPF.cpp:90-172, LambertianBRDF.cpp:44-93,
//                                                GeometricUtilities.cpp:85-98
//   * point on a mesh luminary                  TriangleMeshGeometryIndexed.cpp:207-218,
//                                                GeometricUtilities.cpp:543-569
//   * power heuristic, Russian roulette         PathTransportUtilities.h:86-110, :251
// Random numbers are the same counter-based hash the device uses, so a pixel
// sample follows the same decisions here and on the GPU up to rounding.
// Loaded only by tests and bench.py's CPU-baseline leg.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

const double kPi = 3.14159265358979323846;
const double kInvPi = 1.0 / kPi;
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

struct V { double x, y, z; };
inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator*(V a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V operator-(V a) { return {-a.x, -a.y, -a.z}; }
inline double Dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V Cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V Norm(V a) { return a * (1.0 / std::sqrt(Dot(a, a))); }

struct Light {
    int first, count, emit;
    double area, pdf;
};
struct LTri {
    V v0, e1, e2;
    double cdf;
};

struct Scene {
    const float* tri9;
    std::vector<int> triMesh;
    const int64_t* meshes;
    const float* spectra;
    const int32_t* mi;
    const float* mf;
    const double* cie;
    std::vector<Light> lights;
    std::vector<LTri> ltris;
    std::vector<int> meshLight;
    orc_bvh* bvh;
    int env, envVisible;
    double lmin, lmax, rrThreshold, ynorm;
    int width, height, maxDepth, rrMinDepth, neePerLambda;
    uint32_t seed;
    V pos, fwd, right, up;
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

inline double Spec(const Scene& S, int id, double nm)
{
    int i, j;
    double w;
    if (id < 0 || !Interp(nm, i, j, w)) return 0.0;
    const float* s = S.spectra + 81 * (size_t)id;
    return (double)s[i] + w * ((double)s[j] - (double)s[i]);
}

inline double PowerHeuristic(double a, double b) { return a * a / (a * a + b * b); }

void Sample(const Scene& S, uint32_t pixel, uint32_t sample, double xyz[3])
{
    const uint32_t key = PathKey(S.seed, pixel, sample);
    const int px = (int)(pixel % (uint32_t)S.width), py = (int)(pixel / (uint32_t)S.width);
    const double fx = px + Rand(key, 0), fy = py + Rand(key, 1);
    const double sx = 2.0 * fx / S.width - 1.0, sy = 1.0 - 2.0 * fy / S.height;
    V d = Norm(S.fwd + S.right * sx + S.up * sy);
    V o = S.pos;
    const double hero = S.lmin + Rand(key, 2) * (S.lmax - S.lmin);
    double lam[4];
    const double range = S.lmax - S.lmin;
    lam[0] = hero;
    for (int i = 1; i < 4; ++i) lam[i] = S.lmin + std::fmod(hero - S.lmin + i * range / 4.0, range);
    double thr[4] = {1, 1, 1, 1}, L[4] = {0, 0, 0, 0};
    double bsdfPdf = 0.0;
    for (int depth = 0; depth < S.maxDepth; ++depth) {
        double mx = 0.0;
        bool bad = false;
        for (double v : thr) { if (!std::isfinite(v)) bad = true; mx = std::max(mx, std::fabs(v)); }
        if (bad || mx > 1e6) break;
        const double od[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        double t;
        const int prim = orc_closest_d(S.bvh, od, dd, &t);
        if (prim < 0) {
            if (S.env >= 0 && (depth > 0 || S.envVisible))
                for (int k = 0; k < 4; ++k) L[k] += thr[k] * Spec(S, S.env, lam[k]);
            break;
        }
        const V p = o + d * t;
        const float* tv = S.tri9 + 9 * (size_t)prim;
        const V a = {tv[0], tv[1], tv[2]}, b = {tv[3], tv[4], tv[5]}, c = {tv[6], tv[7], tv[8]};
        V ng = Norm(Cross(b - a, c - a));
        const int mesh = S.triMesh[prim];
        const int mat = (int)S.meshes[4 * mesh + 2];
        const bool ds = S.meshes[4 * mesh + 3] != 0;
        const int light = S.meshLight[mesh];
        if (ds && Dot(ng, d) > 0) ng = -ng;
        const int type = S.mi[5 * mat], refl = S.mi[5 * mat + 1], emit = S.mi[5 * mat + 2];
        // Emission with MIS (:4424-4518).
        if (emit >= 0 && Dot(-d, ng) > 0) {
            double w = 1.0;
            if (bsdfPdf > 0 && light >= 0) {
                const Light& lg = S.lights[light];
                const double cosL = std::fabs(Dot(d, ng));
                if (cosL > 0 && lg.area > 0) w = PowerHeuristic(bsdfPdf, lg.pdf * t * t / (lg.area * cosL));
            }
            for (int k = 0; k < 4; ++k) L[k] += thr[k] * Spec(S, emit, lam[k]) * w;
        }
        if (type != 0) break;
        const V ns = ng;
        const double viewCos = Dot(-d, ns);
        // NEE (LightSampler.cpp:2083-2271), one light sample per wavelength
        // (PathTracingIntegrator.cpp:4528-4549) or one shared sample.
        if (!S.lights.empty() && viewCos > kNearZero) {
            const int nsamp = S.neePerLambda ? 4 : 1;
            for (int k = 0; k < nsamp; ++k) {
                const double ul = Rand(key, Dim(depth, 4 * k));
                int li = 0;
                double acc = 0.0;
                for (li = 0; li < (int)S.lights.size() - 1; ++li) {
                    acc += S.lights[li].pdf;
                    if (ul < acc) break;
                }
                if (li == light) continue;
                const Light& lg = S.lights[li];
                const double ux = Rand(key, Dim(depth, 4 * k + 1)), uy = Rand(key, Dim(depth, 4 * k + 2)),
                             uz = Rand(key, Dim(depth, 4 * k + 3));
                int ts = lg.first + lg.count - 1;
                for (int q = lg.first; q < lg.first + lg.count; ++q)
                    if (S.ltris[q].cdf >= uz) { ts = q; break; }
                const LTri& lt = S.ltris[ts];
                const double sa = std::sqrt(1.0 - ux);
                const double alpha = 1.0 - sa, beta = sa * uy;
                const V pl = lt.v0 + lt.e1 * alpha + lt.e2 * beta;
                const V nl = Norm(Cross(lt.e1, lt.e2));
                V toL = pl - p;
                const double dist = std::sqrt(Dot(toL, toL));
                toL = toL * (1.0 / dist);
                const double cosS = Dot(toL, ns), cosL = Dot(-toL, nl);
                if (cosL <= 0 || cosS <= 0) continue;
                const double pd[3] = {p.x, p.y, p.z}, ld[3] = {toL.x, toL.y, toL.z};
                if (orc_any_d(S.bvh, pd, ld, dist - 0.001)) continue;
                const double geom = lg.area * cosL / (dist * dist);
                const double w = PowerHeuristic(lg.pdf * dist * dist / (lg.area * cosL), cosS * kInvPi) / lg.pdf;
                for (int j = 0; j < 4; ++j) {
                    if (S.neePerLambda && j != k) continue;
                    L[j] += thr[j] * Spec(S, lg.emit, lam[j]) * cosS * geom * Spec(S, refl, lam[j]) * kInvPi * w;
                }
            }
        }
        // Hero BSDF sample (:4597-4719).
        const double u1 = Rand(key, Dim(depth, 16)), u2 = Rand(key, Dim(depth, 17));
        const V w = Dot(d, ns) > kNearZero ? -ns : ns;
        // The cosine lobe is symmetric about w, so any frame gives the same
        // distribution; the device's frame (Duff et al., JCGT 6(1), 2017) is
        // used so that equal random numbers give equal directions.
        const double sg = std::copysign(1.0, w.z);
        const double ia = -1.0 / (sg + w.z);
        const double bb = w.x * w.y * ia;
        const V tx = {1.0 + sg * w.x * w.x * ia, sg * bb, -sg * w.x};
        const V ty = {bb, sg + w.y * w.y * ia, -w.y};
        const double phi = 2.0 * kPi * u1, sint = std::sqrt(u2), cost = std::sqrt(1.0 - u2);
        const V nd = Norm(tx * (std::cos(phi) * sint) + ty * (std::sin(phi) * sint) + w * cost);
        const double pdf = std::fabs(Dot(nd, w)) * kInvPi;
        const V gn = Dot(ng, d) < 0 ? ng : -ng;
        if (!(Dot(nd, gn) > 0)) break;
        double kray[4];
        for (int k = 0; k < 4; ++k) kray[k] = Spec(S, refl, lam[k]);
        double prevMax = 0, currMax = 0;
        for (int k = 0; k < 4; ++k) {
            prevMax = std::max(prevMax, std::fabs(thr[k]));
            currMax = std::max(currMax, std::fabs(thr[k] * kray[k]));
        }
        if (currMax <= kNearZero) break;
        if (depth >= S.rrMinDepth) {
            const double prob = std::min(1.0, currMax / std::max(prevMax, S.rrThreshold));
            if (Rand(key, Dim(depth, 19)) >= prob) break;
            if (prob > 0 && prob < 1)
                for (double& k : kray) k /= prob;
        }
        if (depth + 1 >= S.maxDepth) break;
        for (int k = 0; k < 4; ++k) thr[k] *= kray[k];
        bsdfPdf = pdf;
        o = p + nd * 1e-8;   // Ray::Advance(1e-8), PathTracingIntegrator.cpp:4812
        d = nd;
    }
    xyz[0] = xyz[1] = xyz[2] = 0.0;
    int active = 0;
    for (int k = 0; k < 4; ++k) {
        int i, j;
        double wgt;
        if (!Interp(lam[k], i, j, wgt)) continue;
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

extern "C" int orc_pt_render(const float* tri9, int64_t n_tri, const int64_t* meshes, int32_t n_mesh,
                             const float* spectra, int32_t n_spec, const int32_t* mats_i, const float* mats_f,
                             int32_t n_mat, const int32_t* envi, const double* cam, const double* setd,
                             const int32_t* seti, int32_t spp, int32_t sample_begin, int32_t x0, int32_t y0,
                             int32_t x1, int32_t y1, int32_t threads, double* xyz, const double* cie)
{
    (void)n_spec;
    (void)mats_f;
    Scene S;
    S.tri9 = tri9;
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
    // (b - a) / k_y with k_y the trapezoid integral over whole 5 nm cells
    // (ColorUtils.cpp:327-348).
    {
        const double lo = std::max(S.lmin, 380.0), hi = std::min(S.lmax, 780.0);
        const int f = (int)((lo - 380.0) / 5.0), l = (int)((hi - 380.0) / 5.0);
        double ky = 0.0;
        for (int i = f; i < l; ++i) ky += 0.5 * (cie[81 + i] + cie[81 + i + 1]) * 5.0;
        S.ynorm = ky > 0 ? (S.lmax - S.lmin) / ky : 0.0;
    }
    // Camera frame: forward, right = forward x up, true up = right x forward.
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
        for (int k = 0; k < 81; ++k) mean += spectra[81 * (size_t)emit + k];
        mean /= 81.0;
        weight.push_back(area * std::max(mean, 1e-12));
        S.meshLight[m] = (int)S.lights.size();
        S.lights.push_back(lg);
    }
    double wsum = 0.0;
    for (double w : weight) wsum += w;
    for (size_t i = 0; i < S.lights.size(); ++i) S.lights[i].pdf = weight[i] / wsum;
    S.bvh = orc_bvh_build(tri9, n_tri);
    const int cw = x1 - x0, ch = y1 - y0;
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            const int row = next.fetch_add(1);
            if (row >= ch) break;
            for (int x = 0; x < cw; ++x) {
                const uint32_t pixel = (uint32_t)((y0 + row) * S.width + (x0 + x));
                double acc[3] = {0, 0, 0};
                for (int s = 0; s < spp; ++s) {
                    double v[3];
                    Sample(S, pixel, (uint32_t)(sample_begin + s), v);
                    for (int c = 0; c < 3; ++c) acc[c] += v[c];
                }
                for (int c = 0; c < 3; ++c) xyz[3 * ((size_t)row * cw + x) + c] = acc[c] / spp;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    orc_bvh_destroy(S.bvh);
    return 0;
}
