// Film resolve to colour on the device: the rasterizer's per-pixel XYZ ->
// linear Rec.709 conversion (RISEPel(XYZPel): ColorUtils::XYZtoRec709RGB,
// Utilities/Color/Color.cpp:214-228, with the chromaticity gamut move of
// ColorUtils::MoveXYZIntoRec709RGBGamut, Utilities/Color/ColorUtils.cpp:135-260,351-363)
// and the 8-bit LDR output encode (DisplayTransformWriter::WriteColor,
// Rendering/DisplayTransformWriter.cpp:45-62, the tone curves of
// Rendering/DisplayTransform.h:80-222, and the writers'
// Integerize<sRGBPel>, Utilities/Color/Color_Template.h:128-134 with
// ColorUtils::SRGBTransferFunction, Utilities/Color/ColorUtils.cpp:21-32).
//
// Double precision throughout, built with -fmad=false so every product and
// sum rounds as the host restatement's does.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/rtb200.h"
#include "pathtrace.h"

namespace rtb200 {
namespace {

struct Xy {
    double x, y;
};

// Rec.709 primaries and D65 white point in CIE xy.
__device__ __forceinline__ Xy Red() { return {0.640, 0.330}; }
__device__ __forceinline__ Xy Green() { return {0.300, 0.600}; }
__device__ __forceinline__ Xy Blue() { return {0.150, 0.060}; }
__device__ __forceinline__ Xy White() { return {0.3127, 0.3290}; }

constexpr double kNearZero = 1e-12;

// Where the line a0 -> a1 meets the line b0 -> b1; false when the two are
// parallel to within 1e-12.
__device__ bool Meet(Xy a0, Xy a1, Xy b0, Xy b1, Xy& at)
{
    const double den = (b1.y - b0.y) * (a1.x - a0.x) - (b1.x - b0.x) * (a1.y - a0.y);
    if (den > -kNearZero && den < kNearZero) return false;
    const double ua = ((b1.x - b0.x) * (a0.y - b0.y) - (b1.y - b0.y) * (a0.x - b0.x)) / den;
    at.x = a0.x + ua * (a1.x - a0.x);
    at.y = a0.y + ua * (a1.y - a0.y);
    return true;
}

// p lies strictly between s0 and s1, judged by the x coordinate alone (as
// the reference judges it).
__device__ bool Between(Xy s0, Xy s1, Xy p)
{
    const double v = (p.x - s0.x) / (s1.x - s0.x);
    return v >= kNearZero && v <= 1.0 - kNearZero;
}

// The ray from the white point through c against the gamut edge a-b: true
// with the point to use (c itself when it lies inside that edge).
__device__ bool ClipEdge(Xy c, Xy a, Xy b, Xy& at)
{
    if (!Meet(White(), c, a, b, at) || !Between(a, b, at)) return false;
    if (Between(White(), at, c)) {
        at = c;
        return true;
    }
    return Between(White(), c, at);
}

__device__ void XyzToRec709(const double in[3], double rgb[3])
{
    double X = in[0], Y = in[1], Z = in[2];
    const double inv = 1.0 / (X + Y + Z);
    const Xy c = {X * inv, Y * inv};
    Xy at;
    if (ClipEdge(c, Red(), Green(), at) || ClipEdge(c, Red(), Blue(), at) || ClipEdge(c, Blue(), Green(), at)) {
        const double k = 1.0 / at.y * Y;
        X = k * at.x;
        Z = k * (1.0 - at.x - at.y);
    }
    rgb[0] = 3.240479 * X + -1.537150 * Y + -0.498535 * Z;
    rgb[1] = -0.969256 * X + 1.875992 * Y + 0.041556 * Z;
    rgb[2] = 0.055648 * X + -0.204043 * Y + 1.057311 * Z;
}

__device__ double Sanitise(double x) { return (isfinite(x) && x > 0.0) ? x : 0.0; }
__device__ double Unit(double y) { return fmin(fmax(y, 0.0), 1.0); }

__device__ double HableCurve(double v)
{
    const double A = 0.15, B = 0.50, C = 0.10, D = 0.20, E = 0.02, F = 0.30;
    return ((v * (A * v + C * B) + D * E) / (v * (A * v + B) + D * F)) - E / F;
}

// RTB200_TONE_* curves (public formulas: Reinhard; Narkowicz's ACES fit;
// a log10 sigmoid; Hable's filmic curve with white point 11.2).
__device__ double Tone(int tone, double x)
{
    const double s = Sanitise(x);
    switch (tone) {
    case RTB200_TONE_REINHARD: return s / (1.0 + s);
    case RTB200_TONE_ACES: return Unit(s * (2.51 * s + 0.03) / (s * (2.43 * s + 0.59) + 0.14));
    case RTB200_TONE_AGX: return Unit(0.5 + 0.5 * tanh(1.0 * (log10(s + 1e-10) - 0.0)));
    case RTB200_TONE_HABLE: return Unit(HableCurve(s * 2.0) / HableCurve(11.2));
    default: return s;
    }
}

// sRGB encode, clamp to [0, 1], scale to 255 and truncate.
__device__ unsigned char Encode8(double x)
{
    double v;
    if (x == 0.0) v = 0.0;
    else if (x <= 0.003040247678) v = 12.92 * x;
    else v = 1.055 * pow(x, 1.0 / 2.4) - 0.055;
    if (v > 1.0) v = 1.0;
    if (v < 0.0) v = 0.0;
    return (unsigned char)(v * 255.0);
}

__device__ __forceinline__ double Acc(const float* __restrict__ sum, const float* __restrict__ comp,
                                      const double* __restrict__ wide, size_t k)
{
    return wide ? wide[k] : (double)sum[k] - (double)comp[k];
}

__global__ void KResolveColor(const float* __restrict__ sum, const float* __restrict__ comp,
                              const double* __restrict__ wide, const unsigned* __restrict__ counts, int channels,
                              double inv_spp, int npix, double ev_mul, int tone, float* __restrict__ rgb,
                              unsigned char* __restrict__ rgb8)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        // The pixel's XYZ as rtb200_job_read_film returns it (FP32).
        double xyz[3];
        if (channels == 3) {
            const unsigned c = counts ? counts[p] : 1u;
            for (int k = 0; k < 3; ++k) {
                const double a = Acc(sum, comp, wide, 3 * (size_t)p + k);
                xyz[k] = counts ? (c ? (double)(float)(a / (double)c) : 0.0) : (double)(float)(a * inv_spp);
            }
        } else {
            const double w = Acc(sum, comp, wide, 4 * (size_t)p + 3);
            for (int k = 0; k < 3; ++k)
                xyz[k] = fabs(w) > 1e-10 ? (double)(float)(Acc(sum, comp, wide, 4 * (size_t)p + k) / w) : 0.0;
        }
        double r[3];
        XyzToRec709(xyz, r);
        if (rgb) {
            for (int k = 0; k < 3; ++k) rgb[3 * (size_t)p + k] = (float)r[k];
        } else {
            for (int k = 0; k < 3; ++k) rgb8[3 * (size_t)p + k] = Encode8(Tone(tone, r[k] * ev_mul));
        }
    }
}

}  // namespace

cudaError_t PtResolveColor(const float* sum, const float* comp, const double* wide, const unsigned* counts,
                           int channels, double inv_spp, int npix, double ev_mul, int tone, float* rgb,
                           unsigned char* rgb8, int sms, cudaStream_t st)
{
    if (npix <= 0) return cudaSuccess;
    KResolveColor<<<std::min(sms * 8, (npix + 255) / 256), 256, 0, st>>>(sum, comp, wide, counts, channels, inv_spp,
                                                                         npix, ev_mul, tone, rgb, rgb8);
    return cudaGetLastError();
}

}  // namespace rtb200
