// ref_pt_harness.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// A thin C-ABI harness around the reference renderer's own building blocks of
// the spectral path tracer, so the oracle's restatement of each can be checked
// against the reference's code on the same inputs:
//   * hero + companion wavelengths     Utilities/Color/SampledWavelengths.h:79-106
//   * CIE 1931 lookup, Y integral      Utilities/Color/ColorUtils.cpp:270-348
//   * GGX D, Lambda, G2, VNDF          Utilities/MicrofacetUtils.h:66-371
//   * energy tables, multiple-scattering lobe sampler and pdf, Fresnel average,
//     F_ms                             Utilities/MicrofacetEnergyLUT.h
//   * conductor / dielectric Fresnel   Utilities/Optics.hpp, Utilities/Optics.cpp:101-160
//   * Russian roulette, power heuristic  Utilities/PathTransportUtilities.h:86-110, :251
// The recipe in oracle/Makefile compiles this file with the reference headers
// and ColorUtils.cpp / Color.cpp where they lie (never copied into this
// repository) into oracle/_ref/libref_pt.so.  Only tests load it.

// The reference headers are order-dependent: ColorUtils.h comes last.
#include "Utilities/Color/SampledWavelengths.h"
#include "Utilities/MicrofacetUtils.h"
#include "Utilities/MicrofacetEnergyLUT.h"
#include "Utilities/Optics.h"
#include "Utilities/OrthonormalBasis3D.h"
#include "Utilities/PathTransportUtilities.h"
#include "Utilities/Color/ColorUtils.h"
#include "Interfaces/ILog.h"
#include "Interfaces/IOptions.h"
#include "Sampling/GaussianPixelFilter.h"
#include "Rendering/DisplayTransform.h"
#include "Lights/LightSampler.h"
#include "Lights/LightBVH.h"
#include "Utilities/Color/RGBSpectra.h"
#include "Interfaces/IFunction2D.h"
#include "Utilities/PiecewiseLinearFunction.h"
#include "Utilities/Color/SpectralPacket.h"
#include "Sampling/SobolSequence.h"

namespace RISE
{
	// Optics.cpp reports total internal reflection through GlobalLog(); the
	// harness does not link the reference's log subsystem.
	class QuietPtLog : public ILog
	{
	public:
		void Print( LOG_ENUM, const char* ) const override {}
		void PrintEx( LOG_ENUM, const char*, ... ) const override {}
		void PrintNew( const void*, const char*, const int, const char* ) const override {}
		void PrintNew( const IReference*, const char*, const int, const char* ) const override {}
		void PrintDelete( const void*, const char*, const int ) const override {}
		void PrintDelete( const IReference*, const char*, const int ) const override {}
		void FlushPrinters() override {}
	};
	ILog* GlobalLog() { static QuietPtLog log; return &log; }

	// Default-valued options: the reference-counting base of the pixel
	// filter links the reference's thread wrapper, which reads one
	// scheduling option; the harness does not link the options-file parser.
	class DefaultPtOptions : public IOptions
	{
	public:
		void addref() const override {}
		bool release() const override { return false; }
		unsigned int refcount() const override { return 1; }
		int ReadInt( const char*, int d ) override { return d; }
		double ReadDouble( const char*, double d ) override { return d; }
		bool ReadBool( const char*, bool d ) override { return d; }
		String ReadString( const char*, String d ) override { return d; }
	};
	IOptions& GlobalOptions() { static DefaultPtOptions o; return o; }
}

using namespace RISE;

// The baked table the reference's singleton would load is generated code
// that the harness does not build; tables are loaded from memory instead.
namespace RISE
{
	extern const unsigned int kSpectrumLUTResolution = 0;
	extern const unsigned int kSpectrumLUTNumFloats = 0;
	extern const float kSpectrumLUTFloats[1] = {0.0f};
}

namespace {
inline Vector3 V(const double* p) { return Vector3(p[0], p[1], p[2]); }
inline void Put(const Vector3& v, double* p) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
}  // namespace

extern "C" {

void ref_pt_sample_wavelengths(double u, double lmin, double lmax, double* lam4)
{
    const SampledWavelengths s = SampledWavelengths::SampleEquidistant(u, lmin, lmax);
    for (int i = 0; i < 4; ++i) lam4[i] = s.lambda[i];
}

int ref_pt_xyz_from_nm(double nm, double* xyz3)
{
    XYZPel p(0, 0, 0);
    const bool ok = ColorUtils::XYZFromNM(p, nm);
    xyz3[0] = p.X; xyz3[1] = p.Y; xyz3[2] = p.Z;
    return ok ? 1 : 0;
}

double ref_pt_cie_y_integral(double a, double b) { return ColorUtils::CIE_Y_Integral(a, b); }

double ref_pt_ggx_d(double alpha, double cosH) { return MicrofacetUtils::GGX_D<Scalar>(alpha, cosH); }
double ref_pt_ggx_lambda(double alpha, double cosT) { return MicrofacetUtils::GGX_Lambda(alpha, cosT); }
double ref_pt_ggx_g2(double alpha, double ci, double co) { return MicrofacetUtils::GGX_G2(alpha, ci, co); }

// Visible-normal sample in the reference frame built from n (CreateFromW);
// the frame is returned so the restatement can sample in the same frame.
void ref_pt_vndf_sample(const double* wi, const double* n, double alpha, double u1, double u2, double* m,
                        double* onb9)
{
    OrthonormalBasis3D onb;
    onb.CreateFromW(V(n));
    Put(MicrofacetUtils::VNDF_Sample_Aniso(V(wi), onb, alpha, alpha, u1, u2), m);
    Put(onb.u(), onb9);
    Put(onb.v(), onb9 + 3);
    Put(onb.w(), onb9 + 6);
}

double ref_pt_vndf_pdf(const double* wi, const double* wo, const double* n, double alpha)
{
    OrthonormalBasis3D onb;
    onb.CreateFromW(V(n));
    return MicrofacetUtils::VNDF_Pdf_Aniso(V(wi), V(wo), onb, alpha, alpha);
}

double ref_pt_conductor_f(const double* v, const double* n, double ni, double nt, double k)
{
    return Optics::CalculateConductorReflectance<Scalar>(V(v), V(n), ni, nt, k);
}

double ref_pt_dielectric_r(const double* v, const double* tv, const double* n, double ni, double nt)
{
    return Optics::CalculateDielectricReflectance(V(v), V(tv), V(n), ni, nt);
}

double ref_pt_lookup_ess(double c, double alpha) { return MicrofacetEnergyLUT::LookupEss(c, alpha); }
double ref_pt_lookup_eavg(double alpha) { return MicrofacetEnergyLUT::LookupEavg(alpha); }
double ref_pt_ms_z(double alpha) { return MicrofacetEnergyLUT::MSLobeZ(alpha); }
double ref_pt_ms_pdf(double c, double alpha, double z) { return MicrofacetEnergyLUT::MSPdf(c, alpha, z); }
double ref_pt_ms_sample_cos(double alpha, double u) { return MicrofacetEnergyLUT::SampleMSCosTheta(alpha, u); }

double ref_pt_fresnel_avg(double ni, double nt, double k)
{
    return MicrofacetEnergyLUT::ComputeFresnelAvg<Scalar>(Vector3(0, 0, 1), ni, nt, k);
}

double ref_pt_fms(double favg, double eavg) { return MicrofacetEnergyLUT::ComputeFms<Scalar>(favg, eavg); }

void ref_pt_tables(double* ess, double* eavg)
{
    for (int a = 0; a < MicrofacetEnergyLUT::LUT_SIZE; ++a) {
        for (int c = 0; c < MicrofacetEnergyLUT::LUT_SIZE; ++c)
            ess[a * MicrofacetEnergyLUT::LUT_SIZE + c] = MicrofacetEnergyLUT::E_ss_TABLE[a][c];
        eavg[a] = MicrofacetEnergyLUT::E_avg_TABLE[a];
    }
}

double ref_pt_power_heuristic(double a, double b) { return PathTransportUtilities::PowerHeuristic(a, b); }

int ref_pt_russian_roulette(unsigned depth, unsigned min_depth, double threshold, double cur, double prev, double u,
                            double* survival)
{
    const PathTransportUtilities::RussianRouletteResult r =
        PathTransportUtilities::EvaluateRussianRoulette(depth, min_depth, threshold, cur, prev, u);
    *survival = r.survivalProb;
    return r.terminate ? 1 : 0;
}

// Per-pixel resolve of the rasterizer: RISEPel(XYZPel), the reference's
// XYZ -> linear Rec.709 conversion with its chromaticity gamut move.
void ref_pt_xyz_to_rec709(const double* xyz, double* rgb)
{
    const Rec709RGBPel r = ColorUtils::XYZtoRec709RGB(XYZPel(xyz[0], xyz[1], xyz[2]));
    rgb[0] = r.r; rgb[1] = r.g; rgb[2] = r.b;
}

// LDR output of one pixel: DisplayTransformWriter::WriteColor's exposure
// scale and tone curve, then the 8-bit writers' Integerize<sRGBPel>.
void ref_pt_display(const double* rgb, double exposure_ev, int tone, unsigned char* out3)
{
    const double mul = std::pow(2.0, exposure_ev);
    RISEPel scaled;
    scaled.r = rgb[0] * mul; scaled.g = rgb[1] * mul; scaled.b = rgb[2] * mul;
    const RISEPel mapped = DisplayTransforms::Apply((DISPLAY_TRANSFORM)tone, scaled);
    const RISEColor c(mapped, 1.0);
    const RGBA8 p = c.Integerize<sRGBPel, unsigned char>(255.0);
    out3[0] = p.r; out3[1] = p.g; out3[2] = p.b;
}

// A spectral painter's spectrum as Job::AddSpectralColorPainter builds it
// (piecewise-linear control points sampled into a SpectralPacket of n bins),
// read back at the query wavelengths with SpectralPacket::ValueAtNM.  Query
// wavelengths must lie below the packet's end (ValueAtNM reads one past its
// bins there).
void ref_pt_spectral_packet(const double* nm, const double* amp, int n, double begin, double end,
                            const double* query, int nq, double* out)
{
    Implementation::PiecewiseLinearFunction1D* f = new Implementation::PiecewiseLinearFunction1D();
    for (int i = 0; i < n; ++i) f->addControlPoint(std::make_pair(nm[i], amp[i]));
    const SpectralPacket packet(begin, end, (unsigned)n, f);
    for (int i = 0; i < nq; ++i) out[i] = packet.ValueAtNM(query[i]);
    f->release();
}

// The reference's light BVH over point-like entries (no luminary objects:
// each entry's box is its position, widened by EnsureBoxHasVolume), sampled
// and evaluated at the query points.
void ref_pt_light_bvh(int n, const double* pos, const double* power, int m, const double* pts, const double* xi,
                      int* picked, double* pdf, double* pdf_all)
{
    std::vector<Implementation::LightEntry> entries(n);
    for (int i = 0; i < n; ++i) {
        entries[i].pLight = 0;
        entries[i].lumIndex = 0xFFFFFFFFu;
        entries[i].exitance = power[i];
        entries[i].position = Point3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    }
    Implementation::LuminaryManager::LuminariesList none;
    Implementation::LightBVH bvh;
    bvh.Build(entries, none);
    for (int q = 0; q < m; ++q) {
        const Point3 p(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        Scalar pd = 0;
        picked[q] = (int)bvh.Sample(p, Vector3(0, 1, 0), xi[q], pd);
        pdf[q] = pd;
        for (int i = 0; i < n; ++i) pdf_all[(size_t)q * n + i] = bvh.Pdf((unsigned)i, p, Vector3(0, 1, 0));
    }
}

// RGB -> spectrum with the reference's table code over a table given in
// memory (the body of its generator's .coeff file): the albedo sigmoid's
// coefficients, and the spectrum of the given kind (0 albedo, 1 unbounded)
// at the query wavelengths.
int ref_pt_rgb_uplift(const float* table, unsigned n_floats, const double* rgb, int kind, const double* nm, int nq,
                      double* coeffs, double* values)
{
    static RGBToSpectrumTable t;
    static const float* loaded = nullptr;
    if (loaded != table) {
        if (!t.LoadFromMemory(64, table, n_floats)) return 0;
        loaded = table;
    }
    const RISEPel p(rgb[0], rgb[1], rgb[2]);
    const RGBSigmoidPolynomial poly = t(LUTTargetPel(p));
    coeffs[0] = poly.c0; coeffs[1] = poly.c1; coeffs[2] = poly.c2;
    if (kind == 0) {
        const RGBAlbedoSpectrum s = RGBAlbedoSpectrum::FromRGB(p, t);
        for (int i = 0; i < nq; ++i) values[i] = s.Eval(nm[i]);
    } else {
        const RGBUnboundedSpectrum s = RGBUnboundedSpectrum::FromRGB(p, t);
        for (int i = 0; i < nq; ++i) values[i] = s.Eval(nm[i]);
    }
    return 1;
}

double ref_pt_gaussian_weight(double size, double sigma, double dx, double dy)
{
    Implementation::GaussianPixelFilter* f = new Implementation::GaussianPixelFilter(size, sigma);
    const double w = f->EvaluateFilter(dx, dy);
    f->release();
    return w;
}

// The reference's padded Owen-scrambled Sobol: out[i] = the 32-bit
// scrambled value of SobolSequence::Sample(index[i], dim[i], seed[i]) (its
// double is this value / 2^32), and HashCombine(a[i], b[i]).
void ref_pt_sobol(const uint32_t* index, const uint32_t* dim, const uint32_t* seed, int64_t n, double* out)
{
    for (int64_t i = 0; i < n; ++i) out[i] = SobolSequence::Sample(index[i], dim[i], seed[i]);
}
void ref_pt_hash_combine(const uint32_t* a, const uint32_t* b, int64_t n, uint32_t* out)
{
    for (int64_t i = 0; i < n; ++i) out[i] = SobolSequence::HashCombine(a[i], b[i]);
}

}  // extern "C"
