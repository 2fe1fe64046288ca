// envmap.cpp -- image environments on the host: the Radiance HDR (RGBE)
// reader, the environment's rotation and its importance-sampling tables.
//
// HdrDecode restates HDRReader (RasterImages/HDRReader.cpp:30-205): the
// "#?RADIANCE" signature, header lines up to the resolution line "-Y h +X w"
// (or "+Y h +X w", rows bottom to top; -X is refused), new-style run-length
// scanlines (2, 2, width) with per-component runs (count > 128: a run of
// count - 128 copies) or flat 4-byte pixels with the old (1, 1, 1, n)
// repeat, and the decode value = 2^(e - 136) (byte + 1/2), black for e = 0.
//
// BuildEnvTables restates EnvironmentSampler::Build
// (Rendering/EnvironmentSampler.cpp:150-225): a 64 x 64 grid over the probe
// image's (s, t); each cell weighs the bilinear RGB at its centre times the
// radiance scale, maximum channel, times sin(theta) / theta (1 below theta
// 1e-6, 0 outside the probe disk); rows accumulate into conditional CDFs,
// row totals into the marginal CDF, all normalised (last entries 1).  The
// tables are built in FP64 like the reference's and stored in FP32.
//
// The rotation is RadianceMap::SetOrientation (Rendering/RadianceMap.h):
// XRotation(x) * YRotation(y) * ZRotation(z) in the reference's Matrix4
// storage and product (Utilities/Math3D/MatricesOps.h:274-319,
// Matrices.h:153-170), applied to directions as Vector3Ops::Transform
// (VectorsOps.h:241-247).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "core.h"
#include "env_map.h"

namespace rtb200 {

namespace {

struct Mat {
    double m[4][4];   // the reference's _rc storage
};

Mat Identity()
{
    Mat a{};
    for (int i = 0; i < 4; ++i) a.m[i][i] = 1.0;
    return a;
}

Mat Rot(int axis, double d)
{
    Mat a = Identity();
    const double S = std::sin(d), C = std::cos(d);
    if (axis == 0) { a.m[1][1] = C; a.m[1][2] = S; a.m[2][1] = -S; a.m[2][2] = C; }
    if (axis == 1) { a.m[2][2] = C; a.m[2][0] = S; a.m[0][2] = -S; a.m[0][0] = C; }
    if (axis == 2) { a.m[0][0] = C; a.m[0][1] = S; a.m[1][0] = -S; a.m[1][1] = C; }
    return a;
}

// operator*(Matrix4, Matrix4): ret._rc = sum_k a._kc b._rk.
Mat Mul(const Mat& a, const Mat& b)
{
    Mat r{};
    for (int rr = 0; rr < 4; ++rr)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a.m[k][c] * b.m[rr][k];
            r.m[rr][c] = s;
        }
    return r;
}

}  // namespace

// World -> map rotation as a row-major 3 x 3 (out_c = sum_r m._rc v_r).
void EnvRotation(const double orient_rad[3], float rot[9])
{
    const Mat m = Mul(Mul(Rot(0, orient_rad[0]), Rot(1, orient_rad[1])), Rot(2, orient_rad[2]));
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) rot[3 * c + r] = (float)m.m[r][c];
}

bool HdrDecode(const uint8_t* p, size_t n, int& width, int& height, std::vector<float>* rgb, std::string& err)
{
    size_t at = 0;
    auto line = [&](std::string& out) {
        out.clear();
        if (at >= n) return false;
        while (at < n && p[at] != '\n') out.push_back((char)p[at++]);
        if (at < n) ++at;
        return true;
    };
    static const char kSig[] = "#?RADIANCE";
    if (n < 10 || std::memcmp(p, kSig, 10) != 0) { err = "RADIANCE signature not found"; return false; }
    std::string ln;
    line(ln);
    bool fmt = false, res = false;
    while (line(ln)) {
        if (ln.compare(0, 6, "FORMAT") == 0) { fmt = true; break; }
    }
    if (!fmt) { err = "no FORMAT line"; return false; }
    while (line(ln)) {
        if (ln.compare(0, 2, "-Y") == 0 || ln.compare(0, 2, "+Y") == 0) { res = true; break; }
    }
    if (!res) { err = "no resolution line"; return false; }
    const bool flipY = ln[0] == '+';
    char ya[4] = {0}, xa[4] = {0};
    long h = 0, w = 0;
    if (std::sscanf(ln.c_str(), "%2s %ld %2s %ld", ya, &h, xa, &w) != 4 || w <= 0 || h <= 0)
        { err = "bad resolution line"; return false; }
    if (xa[0] == '-') { err = "-X (flipped) scanlines are not supported"; return false; }
    if ((unsigned long long)w * (unsigned long long)h > (1ull << 28)) { err = "image too large"; return false; }
    width = (int)w;
    height = (int)h;
    if (!rgb) return true;
    std::vector<uint8_t> px((size_t)w * h * 4, 0);
    auto get = [&](uint8_t& b) {
        if (at >= n) return false;
        b = p[at++];
        return true;
    };
    for (long y = 0; y < h; ++y) {
        const size_t start = (size_t)(flipY ? h - y - 1 : y) * (size_t)w;
        uint8_t col[4];
        for (int k = 0; k < 4; ++k)
            if (!get(col[k])) { err = "truncated scanline"; return false; }
        if (col[0] == 2 && col[1] == 2 && (int8_t)col[2] >= 0) {
            for (int comp = 0; comp < 4; ++comp) {
                long x = 0;
                size_t pos = start;
                while (x < w) {
                    uint8_t num;
                    if (!get(num)) { err = "truncated run"; return false; }
                    const bool run = num > 128;
                    const long len = run ? num - 128 : num;
                    uint8_t val = 0;
                    if (run && !get(val)) { err = "truncated run"; return false; }
                    if (len == 0 || x + len > w) { err = "malformed run-length scanline"; return false; }
                    for (long i = 0; i < len; ++i) {
                        uint8_t b = val;
                        if (!run && !get(b)) { err = "truncated run"; return false; }
                        px[4 * pos + comp] = b;
                        ++pos;
                    }
                    x += len;
                }
            }
        } else {
            size_t pos = start;
            for (long x = 0; x < w; ++x) {
                if (x > 0)
                    for (int k = 0; k < 4; ++k)
                        if (!get(col[k])) { err = "truncated scanline"; return false; }
                if (col[0] == 1 && col[1] == 1 && col[2] == 1) {
                    const long num = col[3];
                    // Repeats the pixel before in memory (the previous row's
                    // last one at a row start), as the reference does.
                    if (num == 0 || num > w - x || pos == 0) { err = "malformed repeat"; return false; }
                    for (long i = 0; i < num; ++i, ++pos) std::memcpy(&px[4 * pos], &px[4 * (pos - 1)], 4);
                    x += num - 1;
                } else {
                    std::memcpy(&px[4 * pos], col, 4);
                    ++pos;
                }
            }
        }
    }
    rgb->resize((size_t)w * h * 3);
    for (size_t i = 0; i < (size_t)w * h; ++i) {
        const uint8_t e = px[4 * i + 3];
        for (int k = 0; k < 3; ++k)
            (*rgb)[3 * i + k] = e == 0 ? 0.0f : (float)(std::ldexp(1.0, (int)e - 136) * (px[4 * i + k] + 0.5));
    }
    return true;
}

void BuildEnvTables(const std::vector<float4>& texels, int width, int height, float scale,
                    std::vector<float>& marginal, std::vector<float>& conditional)
{
    constexpr int R = kEnvCdfRes;
    PtEnvMap E{};
    E.texels = texels.data();
    E.width = width;
    E.height = height;
    std::vector<double> cond((size_t)R * (R + 1)), marg(R + 1);
    for (int v = 0; v < R; ++v) {
        double* row = &cond[(size_t)v * (R + 1)];
        row[0] = 0.0;
        for (int u = 0; u < R; ++u) {
            const double s = (u + 0.5) / R, t = (v + 0.5) / R;
            float rgb[3];
            EnvBilinear(E, (float)s, (float)t, rgb);
            const double lum = std::max({(double)rgb[0], (double)rgb[1], (double)rgb[2]}) * (double)scale;
            const double dx = s - 0.5, dy = -(t - 0.5);
            const double rt = std::sqrt(dx * dx + dy * dy);
            const double th = rt * 6.283185307179586;
            double wgt = th < 1e-6 ? 1.0 : std::sin(th) / th;
            if (rt > 0.5) wgt = 0.0;
            row[u + 1] = row[u] + lum * wgt;
        }
    }
    marg[0] = 0.0;
    for (int v = 0; v < R; ++v) marg[v + 1] = marg[v] + cond[(size_t)v * (R + 1) + R];
    const double total = marg[R];
    marginal.assign(R + 1, 0.0f);
    conditional.assign((size_t)R * (R + 1), 0.0f);
    if (!(total > 0.0)) return;
    for (int v = 0; v < R; ++v) {
        double* row = &cond[(size_t)v * (R + 1)];
        const double rt = row[R];
        for (int u = 0; u <= R; ++u) conditional[(size_t)v * (R + 1) + u] = rt > 0.0 ? (float)(row[u] / rt) : (float)row[u];
        conditional[(size_t)v * (R + 1) + R] = 1.0f;
    }
    for (int v = 0; v <= R; ++v) marginal[v] = (float)(marg[v] / total);
    marginal[R] = 1.0f;
}

}  // namespace rtb200

using namespace rtb200;

extern "C" {

int rtb200_hdr_decode(const uint8_t* bytes, int64_t n, int32_t* width, int32_t* height, float* rgb)
{
    if (!bytes || n <= 0 || !width || !height) return RTB200_E_INVALID;
    int w = 0, h = 0;
    std::string err;
    std::vector<float> img;
    if (!HdrDecode(bytes, (size_t)n, w, h, rgb ? &img : nullptr, err)) return RTB200_E_INVALID;
    *width = w;
    *height = h;
    if (rgb) std::memcpy(rgb, img.data(), img.size() * sizeof(float));
    return RTB200_OK;
}

}  // extern "C"
