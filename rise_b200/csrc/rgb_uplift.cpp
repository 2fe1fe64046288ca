// rgb_uplift.cpp -- RGB to spectrum uplift for the reference's RGB painters:
// the Jakob-Hanika (2019) sigmoid-polynomial table and its lookup.
//
// A spectrum is S(l) = s(c0 t^2 + c1 t + c2), t = (l - 380) / 400 on
// 380..780 nm (0 outside), with the stable sigmoid s(x) = 1/2 + x / (2
// sqrt(1 + x^2)) (RGBSigmoidPolynomial, Utilities/Color/RGBSigmoidPolynomial.h:58-70).
//
// The table follows the reference's generator step for step
// (tools/JakobHanikaLUTGen.cpp, target Rec.709), so its coefficients are
// the reference's: three sub-tables by largest channel, each res^3 cells at
// z = sin^2(pi/2 * i/(res-1)) and linear x, y (the other two channels over
// z); each cell solves for (c0, c1, c2) by Gauss-Newton on the Rec.709
// residual of the spectrum integrated against the CIE 1931 observer under a
// flat illuminant (normalised to Y = 1 for S = 1), with a central-difference
// Jacobian (step 5e-4), Levenberg-Marquardt damping 1e-6 * max diagonal,
// up to 10 halvings of a rejected step, at most 200 iterations, accepted
// below 1e-4; a cell starts from the previous cell of its row (the first
// cell of a row from the first cell of the previous row, the plane's first
// row from zero) and is solved again from zero when that leaves a residual
// above 1e-4; black cells are (0, 0, -100).  Planes of one largest channel
// and one z are independent, so they are solved in parallel.
//
// The lookup (RGBToSpectrumTable::operator(),
// Utilities/Color/RGBToSpectrumTable.cpp:161-243) clamps RGB to [0, 1],
// picks the sub-table of the largest channel, maps z back through
// asin(sqrt(z)) and interpolates the eight surrounding cells trilinearly.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>

#include "cie1931.h"
#include "core.h"

namespace rtb200 {
namespace {

constexpr int kRes = 64;
const double kCx[RTB200_CIE_COUNT] = {RTB200_CIE_XBAR};
const double kCy[RTB200_CIE_COUNT] = {RTB200_CIE_YBAR};
const double kCz[RTB200_CIE_COUNT] = {RTB200_CIE_ZBAR};
// XYZ (D65) -> linear Rec.709 (Utilities/Color/Color.cpp:22-25).
const double kToRgb[3][3] = {{3.240479, -1.537150, -0.498535},
                             {-0.969256, 1.875992, 0.041556},
                             {0.055648, -0.204043, 1.057311}};

inline double Sigmoid(double x) { return 0.5 + x / (2.0 * std::sqrt(1.0 + x * x)); }

// Rec.709 of the sigmoid spectrum c under a flat illuminant.
void Forward(const double c[3], double rgb[3])
{
    double X = 0.0, Y = 0.0, Z = 0.0, yn = 0.0;
    for (int i = 0; i < RTB200_CIE_COUNT; ++i) {
        const double l = 380.0 + i * 5.0;
        const double t = (l - 380.0) * (1.0 / 400.0);
        const double s = Sigmoid(c[0] * t * t + c[1] * t + c[2]);
        X += s * kCx[i];
        Y += s * kCy[i];
        Z += s * kCz[i];
        yn += kCy[i];
    }
    const double inv = 1.0 / yn;
    X *= inv;
    Y *= inv;
    Z *= inv;
    // The chromatic adaptation to the target white is the identity for D65.
    const double Xa = 1.0 * X + 0.0 * Y + 0.0 * Z;
    const double Ya = 0.0 * X + 1.0 * Y + 0.0 * Z;
    const double Za = 0.0 * X + 0.0 * Y + 1.0 * Z;
    for (int k = 0; k < 3; ++k) rgb[k] = kToRgb[k][0] * Xa + kToRgb[k][1] * Ya + kToRgb[k][2] * Za;
}

double Residual(const double c[3], const double target[3], double r[3])
{
    double rgb[3];
    Forward(c, rgb);
    for (int k = 0; k < 3; ++k) r[k] = rgb[k] - target[k];
    return std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

// Gauss-Newton from the seed in c; c ends at the best point met.
double Solve(const double target[3], double c[3])
{
    const double kAccept = 1e-4, kStep = 5e-4;
    double best[3] = {c[0], c[1], c[2]};
    double r[3];
    double bestNorm = Residual(c, target, r);
    for (int iter = 0; iter < 200; ++iter) {
        const double norm = Residual(c, target, r);
        if (norm < bestNorm) {
            bestNorm = norm;
            for (int k = 0; k < 3; ++k) best[k] = c[k];
        }
        if (norm < kAccept) break;
        double J[3][3];
        for (int j = 0; j < 3; ++j) {
            double cp[3] = {c[0], c[1], c[2]}, cm[3] = {c[0], c[1], c[2]};
            cp[j] += kStep;
            cm[j] -= kStep;
            double fp[3], fm[3];
            Forward(cp, fp);
            Forward(cm, fm);
            for (int i = 0; i < 3; ++i) J[i][j] = (fp[i] - fm[i]) / (2.0 * kStep);
        }
        double A[3][3], g[3];
        for (int i = 0; i < 3; ++i) {
            g[i] = J[0][i] * r[0] + J[1][i] * r[1] + J[2][i] * r[2];
            for (int j = 0; j < 3; ++j) A[i][j] = J[0][i] * J[0][j] + J[1][i] * J[1][j] + J[2][i] * J[2][j];
        }
        const double damp = 1e-6 * std::max({A[0][0], A[1][1], A[2][2]});
        for (int i = 0; i < 3; ++i) A[i][i] += damp;
        const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                           A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
        if (std::fabs(det) < 1e-40) break;
        const double id = 1.0 / det;
        double M[3][3];
        M[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id;
        M[0][1] = -(A[0][1] * A[2][2] - A[0][2] * A[2][1]) * id;
        M[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
        M[1][0] = -(A[1][0] * A[2][2] - A[1][2] * A[2][0]) * id;
        M[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
        M[1][2] = -(A[0][0] * A[1][2] - A[0][2] * A[1][0]) * id;
        M[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id;
        M[2][1] = -(A[0][0] * A[2][1] - A[0][1] * A[2][0]) * id;
        M[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
        double step[3];
        for (int i = 0; i < 3; ++i) step[i] = M[i][0] * g[0] + M[i][1] * g[1] + M[i][2] * g[2];
        double h = 1.0;
        bool moved = false;
        for (int ls = 0; ls < 10; ++ls) {
            const double n[3] = {c[0] - h * step[0], c[1] - h * step[1], c[2] - h * step[2]};
            double rn[3];
            const double nn = Residual(n, target, rn);
            if (nn < norm) {
                moved = true;
                for (int k = 0; k < 3; ++k) c[k] = n[k];
                if (nn < bestNorm) {
                    bestNorm = nn;
                    for (int k = 0; k < 3; ++k) best[k] = c[k];
                }
                break;
            }
            h *= 0.5;
        }
        if (!moved) break;
    }
    for (int k = 0; k < 3; ++k) c[k] = best[k];
    return bestNorm;
}

inline double GridZ(int i)
{
    const double t = (double)i / (double)(kRes - 1);
    const double s = std::sin(0.5 * M_PI * t);
    return s * s;
}
inline double GridLin(int i) { return (double)i / (kRes - 1); }

// One (largest channel, z) plane, rows in x, cells in y.
void SolvePlane(int maxc, int iz, float* table)
{
    const double z = GridZ(iz);
    double rowSeed[3] = {0.0, 0.0, 0.0};
    for (int ix = 0; ix < kRes; ++ix) {
        double prev[3] = {rowSeed[0], rowSeed[1], rowSeed[2]};
        for (int iy = 0; iy < kRes; ++iy) {
            double rgb[3];
            rgb[maxc] = z;
            rgb[(maxc + 1) % 3] = GridLin(ix) * z;
            rgb[(maxc + 2) % 3] = GridLin(iy) * z;
            double c[3] = {prev[0], prev[1], prev[2]};
            if (z < 1e-9) {
                c[0] = c[1] = 0.0;
                c[2] = -100.0;
            } else {
                const double res = Solve(rgb, c);
                if (res > 1e-4) {
                    double alt[3] = {0.0, 0.0, 0.0};
                    if (Solve(rgb, alt) < res)
                        for (int k = 0; k < 3; ++k) c[k] = alt[k];
                }
            }
            float* o = table + 3 * ((((size_t)maxc * kRes + iz) * kRes + ix) * kRes + iy);
            for (int k = 0; k < 3; ++k) o[k] = (float)c[k];
            for (int k = 0; k < 3; ++k) prev[k] = c[k];
            if (iy == 0)
                for (int k = 0; k < 3; ++k) rowSeed[k] = c[k];
        }
    }
}

const std::vector<float>& Table()
{
    static std::vector<float> table;
    static std::once_flag once;
    std::call_once(once, []() {
        table.assign(3 * (size_t)3 * kRes * kRes * kRes, 0.0f);
        std::atomic<int> next(0);
        const int nt = (int)std::max(1u, std::thread::hardware_concurrency());
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&]() {
                for (int k; (k = next.fetch_add(1)) < 3 * kRes;) SolvePlane(k / kRes, k % kRes, table.data());
            });
        for (auto& t : pool) t.join();
    });
    return table;
}

inline const float* Cell(const std::vector<float>& T, int maxc, int iz, int ix, int iy)
{
    iz = std::max(0, std::min(kRes - 1, iz));
    ix = std::max(0, std::min(kRes - 1, ix));
    iy = std::max(0, std::min(kRes - 1, iy));
    return T.data() + 3 * ((((size_t)maxc * kRes + iz) * kRes + ix) * kRes + iy);
}

inline float Lerp(float a, float b, double t) { return (float)((double)a * (1.0 - t) + (double)b * t); }

}  // namespace

const std::vector<float>& UpliftTable() { return Table(); }

void RgbToSigmoid(const double rgb_in[3], double c[3])
{
    const std::vector<float>& T = Table();
    double r = std::max(0.0, std::min(1.0, rgb_in[0]));
    double g = std::max(0.0, std::min(1.0, rgb_in[1]));
    double b = std::max(0.0, std::min(1.0, rgb_in[2]));
    int maxc;
    double z, x, y;
    if (r >= g && r >= b) {
        maxc = 0; z = r; x = z > 1e-9 ? g / z : 0.0; y = z > 1e-9 ? b / z : 0.0;
    } else if (g >= r && g >= b) {
        maxc = 1; z = g; x = z > 1e-9 ? b / z : 0.0; y = z > 1e-9 ? r / z : 0.0;
    } else {
        maxc = 2; z = b; x = z > 1e-9 ? r / z : 0.0; y = z > 1e-9 ? g / z : 0.0;
    }
    const double fz = std::max(0.0, std::min((double)(kRes - 1),
                                             std::asin(std::sqrt(std::max(0.0, std::min(1.0, z)))) * (2.0 / M_PI) *
                                                 (kRes - 1)));
    const double fx = std::max(0.0, std::min((double)(kRes - 1), x * (kRes - 1)));
    const double fy = std::max(0.0, std::min((double)(kRes - 1), y * (kRes - 1)));
    const int iz = (int)std::floor(fz), ix = (int)std::floor(fx), iy = (int)std::floor(fy);
    const double tz = fz - iz, tx = fx - ix, ty = fy - iy;
    for (int k = 0; k < 3; ++k) {
        const float a00 = Lerp(Cell(T, maxc, iz, ix, iy)[k], Cell(T, maxc, iz, ix + 1, iy)[k], tx);
        const float a01 = Lerp(Cell(T, maxc, iz + 1, ix, iy)[k], Cell(T, maxc, iz + 1, ix + 1, iy)[k], tx);
        const float a10 = Lerp(Cell(T, maxc, iz, ix, iy + 1)[k], Cell(T, maxc, iz, ix + 1, iy + 1)[k], tx);
        const float a11 = Lerp(Cell(T, maxc, iz + 1, ix, iy + 1)[k], Cell(T, maxc, iz + 1, ix + 1, iy + 1)[k], tx);
        const float b0 = Lerp(a00, a10, ty);
        const float b1 = Lerp(a01, a11, ty);
        c[k] = (double)Lerp(b0, b1, tz);
    }
}

}  // namespace rtb200

using namespace rtb200;

extern "C" {

int rtb200_rgb_uplift(const double* rgb, int32_t kind, double* out)
{
    if (!rgb || !out || (kind != RTB200_RGB_ALBEDO && kind != RTB200_RGB_UNBOUNDED)) return RTB200_E_INVALID;
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(rgb[k])) return RTB200_E_INVALID;
    double scale = 1.0, c[3] = {0.0, 0.0, 0.0};
    if (kind == RTB200_RGB_ALBEDO) {
        RgbToSigmoid(rgb, c);
    } else {
        // RGBUnboundedSpectrum::FromRGB (Utilities/Color/RGBSpectra.h:60-79).
        scale = std::max(rgb[0], std::max(rgb[1], rgb[2]));
        if (scale > 1e-9) {
            const double n[3] = {rgb[0] / scale, rgb[1] / scale, rgb[2] / scale};
            RgbToSigmoid(n, c);
        }
    }
    out[0] = c[0];
    out[1] = c[1];
    out[2] = c[2];
    out[3] = scale;
    return RTB200_OK;
}

int rtb200_rgb_uplift_table(float* coeffs)
{
    if (!coeffs) return RTB200_E_INVALID;
    const std::vector<float>& T = Table();
    std::copy(T.begin(), T.end(), coeffs);
    return RTB200_OK;
}

}  // extern "C"
