// ref_render_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A small C interface over the reference renderer's own library
// (oracle/_ref/librise_ref.so, built by oracle/rise_ref.mk from the
// reference sources in place).  It loads a .RISEscene into a reference job,
// the way the reference's in-process tests do
// (tests/EnvLightBalanceTest.cpp:108-150,209-240: RISE_CreateJobPriv ->
// LoadAsciiSceneViaCst -> replace the outputs with an in-memory capture ->
// Rasterize), and offers two ways to render it:
//
//   rr_render     the reference's whole pipeline (Job::Rasterize through
//                 PixelBasedRasterizerHelper and PathTracingSpectralRasterizer
//                 ::IntegratePixel, Sobol sampling seeded by
//                 HashCombine(x, y)); returns the resolved linear Rec.709
//                 image the rasterizer hands its outputs;
//   rr_integrate  the reference's per-sample function
//                 PathTracingSpectralRasterizer::IntegratePixelSpectral
//                 (camera ray, wavelength bundle, PathTracingIntegrator
//                 ::IntegrateRayHWSS, XYZ with the rasterizer's
//                 normalisation) driven by a box-filter pixel loop of ours
//                 that restates IntegratePixel's (PathTracingSpectral
//                 Rasterizer.cpp:206-479, pixel_filter box of width 1:
//                 screen point (x + u - 1/2, (height - y) + v - 1/2), weight
//                 1, XYZ averaged over the samples), with a batch number
//                 mixed into the Owen-scrambling seed.  Batch 0 uses the
//                 reference's seed HashCombine(x, y) unchanged; batch b > 0
//                 uses HashCombine(HashCombine(x, y), b), so batches are
//                 independent estimates (the reference's own pixel loop
//                 always seeds a pixel the same way).  It returns per-pixel
//                 XYZ, before the film's colour conversion.
//
// Everything is double precision, as in the reference.

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <thread>
#include <vector>

#include "Interfaces/IJob.h"
#include "Interfaces/IJobPriv.h"
#include "Interfaces/IRasterizer.h"
#include "Interfaces/IRasterizerOutput.h"
#include "Interfaces/IRasterImage.h"
#include "Interfaces/IScenePriv.h"
#include "Rendering/PathTracingSpectralRasterizer.h"
#include "Sampling/SobolSequence.h"
#include "Utilities/Color/Color_Template.h"
#include "Utilities/RandomNumbers.h"
#include "Utilities/Reference.h"
#include "Utilities/RuntimeContext.h"
#include "Utilities/SobolSampler.h"
#include "Utilities/IndependentSampler.h"
#include "Utilities/MediaPathLocator.h"

#include <string>

using namespace RISE;
using namespace RISE::Implementation;

namespace {

// The final image the rasterizer hands its outputs, captured in memory.
class CaptureOutput : public virtual IRasterizerOutput, public virtual Reference
{
public:
    std::vector<double> rgb;
    unsigned int width = 0, height = 0;

protected:
    virtual ~CaptureOutput() {}

public:
    void OutputIntermediateImage(const IRasterImage&, const Rect*) override {}
    void OutputImage(const IRasterImage& img, const Rect*, const unsigned int) override
    {
        width = img.GetWidth();
        height = img.GetHeight();
        rgb.assign(size_t(width) * height * 3, 0.0);
        for (unsigned int y = 0; y < height; ++y)
            for (unsigned int x = 0; x < width; ++x) {
                const RISEColor c = img.GetPEL(x, y);
                double* o = &rgb[(size_t(y) * width + x) * 3];
                o[0] = c.base.r;
                o[1] = c.base.g;
                o[2] = c.base.b;
            }
    }
};

// Reaches the rasterizer's per-sample function, which is protected: a
// pointer to it is formed through a derived class, as the language allows.
struct SampleAccess : public PathTracingSpectralRasterizer
{
    typedef XYZPel (PathTracingSpectralRasterizer::*Fn)(const RuntimeContext&, const RasterizerState&,
                                                         const Point2&, const IScene&, ISampler&,
                                                         const IRadianceMap*, PixelAOV*) const;
    static Fn Get() { return &SampleAccess::IntegratePixelSpectral; }
};

struct RefJob
{
    IJobPriv* job = nullptr;
    bool prepared = false;
};

}  // namespace

extern "C" {

// Loads a scene; returns an opaque job or null.  Files the scene names are
// looked up in the scene's folder (added to the reference's media paths).
void* rr_load(const char* scene_path)
{
    {
        std::string dir(scene_path);
        const size_t cut = dir.find_last_of('/');
        dir = cut == std::string::npos ? std::string(".") : dir.substr(0, cut + 1);
        if (dir.back() != '/') dir += '/';
        GlobalMediaPathLocator().AddPath(dir.c_str());
    }
    IJobPriv* job = nullptr;
    if (!RISE_CreateJobPriv(&job) || !job) return nullptr;
    if (!job->LoadAsciiSceneViaCst(scene_path)) {
        safe_release(job);
        return nullptr;
    }
    job->RemoveRasterizerOutputs();
    RefJob* r = new RefJob;
    r->job = job;
    return r;
}

void rr_free(void* h)
{
    RefJob* r = static_cast<RefJob*>(h);
    if (!r) return;
    safe_release(r->job);
    delete r;
}

// Film size of the loaded scene (0 on error).
int rr_size(void* h, unsigned int* width, unsigned int* height)
{
    RefJob* r = static_cast<RefJob*>(h);
    IScenePriv* scene = r ? r->job->GetScene() : nullptr;
    if (!scene || !scene->GetFilm()) return 0;
    *width = scene->GetFilm()->GetWidth();
    *height = scene->GetFilm()->GetHeight();
    return 1;
}

// The reference's whole pipeline; out = width * height * 3 linear Rec.709
// doubles, rows from the top.  Returns 1 on success.
int rr_render(void* h, double* out, unsigned int width, unsigned int height)
{
    RefJob* r = static_cast<RefJob*>(h);
    if (!r) return 0;
    CaptureOutput* cap = new CaptureOutput();
    r->job->GetRasterizer()->AddRasterizerOutput(cap);
    const bool ok = r->job->Rasterize();
    r->job->RemoveRasterizerOutputs();
    r->prepared = true;
    int rc = 0;
    if (ok && cap->width == width && cap->height == height) {
        std::copy(cap->rgb.begin(), cap->rgb.end(), out);
        rc = 1;
    }
    safe_release(cap);
    return rc;
}

// Mean XYZ of `spp` samples per pixel over the rows [y0, y1) and columns
// [x0, x1) through the reference's per-sample function (see the file
// comment).  independent != 0 draws the path's numbers from the reference's
// IndependentSampler over the row's twister instead of its Sobol sampler.  out = (y1 - y0) * (x1 - x0) * 3 doubles.  Camera jitter and the
// hero-wavelength number come from a Mersenne twister per row (the
// reference draws both from its runtime context's twister too).  Returns 1
// on success.
int rr_integrate(void* h, unsigned int x0, unsigned int y0, unsigned int x1, unsigned int y1,
                 unsigned int spp, unsigned int batch, int threads, int independent, double* out)
{
    RefJob* r = static_cast<RefJob*>(h);
    if (!r || x1 <= x0 || y1 <= y0 || spp == 0) return 0;
    IScenePriv* scene = r->job->GetScene();
    PathTracingSpectralRasterizer* rast =
        dynamic_cast<PathTracingSpectralRasterizer*>(r->job->GetRasterizer());
    if (!scene || !rast || !scene->GetCamera() || !scene->GetFilm()) return 0;
    const unsigned int height = scene->GetFilm()->GetHeight();
    if (!r->prepared) {
        // One pixel through the reference's own pass attaches the scene to
        // the ray caster, builds the acceleration structures and the light
        // sampler, and runs the rasterizer's pre-render set-up.
        if (!r->job->RasterizeRegion(0, 0, 0, 0)) return 0;
        r->prepared = true;
    }
    const SampleAccess::Fn fn = SampleAccess::Get();
    const IRadianceMap* radiance = scene->GetGlobalRadianceMap();
    const unsigned int w = x1 - x0;
    std::atomic<unsigned int> next_row(y0);
    auto work = [&]() {
        for (;;) {
            const unsigned int y = next_row.fetch_add(1);
            if (y >= y1) break;
            RandomNumberGenerator rng(0x5bd1e995u ^ (batch * 2654435761u) ^ (y * 40503u + 1u));
            RuntimeContext rc(rng, RuntimeContext::PASS_NORMAL, true);
            rast->PrepareRuntimeContext(rc);
            for (unsigned int x = x0; x < x1; ++x) {
                const RasterizerState rs = {x, y};
                uint32_t seed = SobolSequence::HashCombine(x, y);
                if (batch) seed = SobolSequence::HashCombine(seed, batch);
                double X = 0, Y = 0, Z = 0;
                for (unsigned int s = 0; s < spp; ++s) {
                    const double u = rng.CanonicalRandom(), v = rng.CanonicalRandom();
                    const Point2 pt(double(x) + u - 0.5, double(height - y) + v - 0.5);
                    SobolSampler sobol(s, seed);
                    IndependentSampler indep(rng);
                    ISampler& sampler = independent ? static_cast<ISampler&>(indep) : static_cast<ISampler&>(sobol);
                    rc.pSampler = &sampler;
                    const XYZPel c = (rast->*fn)(rc, rs, pt, *scene, sampler, radiance, nullptr);
                    rc.pSampler = nullptr;
                    X += c.X;
                    Y += c.Y;
                    Z += c.Z;
                }
                double* o = out + (size_t(y - y0) * w + (x - x0)) * 3;
                o[0] = X / spp;
                o[1] = Y / spp;
                o[2] = Z / spp;
            }
        }
    };
    const int n = std::max(1, threads);
    std::vector<std::thread> pool;
    for (int t = 0; t < n; ++t) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    return 1;
}

}  // extern "C"
