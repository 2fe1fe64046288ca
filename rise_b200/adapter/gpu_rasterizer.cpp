// gpu_rasterizer.cpp -- see gpu_rasterizer.h.
#include "gpu_rasterizer.h"

#include <vector>

#include "Interfaces/IProgressCallback.h"
#include "Interfaces/IRasterImage.h"
#include "Interfaces/IRasterizerOutput.h"
#include "RISE_API.h"

namespace RISE {
namespace Implementation {

namespace {

// Passes rtb200's progress reports to the rasterizer's IProgressCallback:
// this pass's fraction placed in the whole render's.
struct ProgressBridge {
    IProgressCallback* cb;
    double base, share, total;
};

int32_t Bridge(void* user, double progress, double total)
{
    const ProgressBridge* b = static_cast<const ProgressBridge*>(user);
    const double f = total > 0.0 ? progress / total : 1.0;
    return b->cb->Progress(b->base + b->share * f, b->total) ? 1 : 0;
}

}  // namespace

GpuPathTracingSpectralRasterizer::GpuPathTracingSpectralRasterizer(const rtb200_render_settings& settings,
                                                                   unsigned int spp_, unsigned int passes_,
                                                                   int device_)
    : base(settings), spp(spp_), passes(passes_ ? passes_ : 1), device(device_)
{
}

GpuPathTracingSpectralRasterizer::~GpuPathTracingSpectralRasterizer()
{
    if (dev_scene) rtb200_scene_destroy(dev_scene);
    if (ctx) rtb200_ctx_destroy(ctx);
}

void GpuPathTracingSpectralRasterizer::AttachToScene(const IScene*) {}

void GpuPathTracingSpectralRasterizer::DetachFromScene(const IScene* pScene)
{
    if (pScene == dev_for && dev_scene) {
        rtb200_scene_destroy(dev_scene);
        dev_scene = nullptr;
        dev_for = nullptr;
    }
}

unsigned int GpuPathTracingSpectralRasterizer::PredictTimeToRasterizeScene(const IScene&, const ISampling2D&,
                                                                          unsigned int* pActualTime) const
{
    if (pActualTime) *pActualTime = 0;
    return 0;
}

void GpuPathTracingSpectralRasterizer::RasterizeScene(const IScene& scene, const Rect* pRect, IRasterizeSequence*) const
{
    auto fail = [&](int rc, const std::string& what) {
        last_status = rc;
        last_message = what + (ctx ? std::string(": ") + rtb200_last_error(ctx) : std::string());
    };
    last_status = RTB200_OK;
    last_message.clear();
    if (!ctx && rtb200_ctx_create(device, 0, &ctx) != RTB200_OK) {
        fail(RTB200_E_DEVICE, "no CUDA device");
        ctx = nullptr;
        return;
    }
    if (dev_for != &scene) {
        if (dev_scene) rtb200_scene_destroy(dev_scene);
        dev_scene = nullptr;
        dev_for = nullptr;
        rtb200_rise::Scene ex;
        rtb200_rise::ExtractScene(scene, ex);
        refused = ex.refused;
        int rc = rtb200_scene_create(ctx, &dev_scene);
        if (!rc) rc = rtb200_rise::UploadScene(ex, dev_scene);
        if (!rc) rc = rtb200_scene_commit(dev_scene, RTB200_BVH_F32);
        if (rc) {
            fail(rc, "scene upload");
            if (dev_scene) rtb200_scene_destroy(dev_scene);
            dev_scene = nullptr;
            return;
        }
        dev_for = &scene;
        job_settings = base;
        job_settings.width = ex.width;
        job_settings.height = ex.height;
        for (int k = 0; k < 3; ++k) {
            job_settings.cam_pos[k] = ex.cam_pos[k];
            job_settings.cam_look[k] = ex.cam_look[k];
            job_settings.cam_up[k] = ex.cam_up[k];
        }
        job_settings.fov_deg = ex.fov_deg;
    }
    rtb200_job* job = nullptr;
    int rc = rtb200_job_create(dev_scene, &job_settings, &job);
    if (rc) {
        fail(rc, "job");
        return;
    }
    ProgressBridge bridge{pProgressFunc, 0.0, 0.0, (double)spp};
    unsigned int done = 0;
    for (unsigned int p = 0; p < passes && done < spp && !rc; ++p) {
        const unsigned int n = (spp - done) / (passes - p);
        if (!n) continue;
        if (pProgressFunc) {
            bridge.base = done;
            bridge.share = n;
            rtb200_job_set_progress(job, Bridge, &bridge);
        }
        rc = rtb200_job_render(job, (int32_t)n);
        done += n;
    }
    if (rc && rc != RTB200_E_CANCELLED) {
        fail(rc, "render");
        rtb200_job_destroy(job);
        return;
    }
    last_status = rc;
    const int w = job_settings.width, h = job_settings.height;
    std::vector<float> rgb((size_t)w * h * 3);
    rc = rtb200_job_read_rgb(job, rgb.data());
    rtb200_job_destroy(job);
    if (rc) {
        fail(rc, "film readback");
        return;
    }
    IRasterImage* img = nullptr;
    RISE_API_CreateRISEColorRasterImage(&img, w, h, RISEColor(0, 0, 0, 0));
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const float* c = &rgb[3 * ((size_t)y * w + x)];
            img->SetPEL(x, y, RISEColor(RISEPel(c[0], c[1], c[2]), 1.0));
        }
    std::lock_guard<std::mutex> g(outsMutex);
    for (IRasterizerOutput* o : outs) o->OutputImage(*img, pRect, 0);
    safe_release(img);
}

void GpuPathTracingSpectralRasterizer::RasterizeSceneAnimation(const IScene& pScene, const Scalar, const Scalar,
                                                               const unsigned int, const bool, const bool,
                                                               const Rect* pRect, const unsigned int*,
                                                               IRasterizeSequence* seq) const
{
    // One frame of a static scene: this path has no time-varying
    // geometry, so every frame is the still image.
    RasterizeScene(pScene, pRect, seq);
}

}  // namespace Implementation
}  // namespace RISE
