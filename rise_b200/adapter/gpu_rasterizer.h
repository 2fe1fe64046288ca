// gpu_rasterizer.h -- a RISE rasterizer (IRasterizer, Interfaces/IRasterizer.h)
// that renders the spectral path tracer's image on the GPU through rtb200:
// the drop-in for PathTracingSpectralRasterizer on this path.  Built inside a
// RISE tree, beside the reference's own rasterizers; a job registers it where
// Job::SetPathTracingSpectralRasterizer (Job.cpp:7984-8085) registers the CPU
// one, with the same settings.
//
// RasterizeScene reads the scene (rise_extract.h), uploads it to a device
// scene on the first call (kept while the same scene is rasterized again),
// renders the settings' samples per pixel as progressive passes, reporting
// progress to the IProgressCallback set on it (a false return stops the
// render at a whole number of samples per pixel), and hands every rasterizer
// output the image as the reference's rasterizers do: linear Rec.709
// RISEColor pixels (the XYZ -> RGB resolve of the film, computed on the
// device), rows from the top, through IRasterizerOutput::OutputImage.
#pragma once

#include "Rendering/Rasterizer.h"
#include "rise_extract.h"
#include "rtb200.h"

namespace RISE {
namespace Implementation {

class GpuPathTracingSpectralRasterizer : public virtual Rasterizer
{
public:
    // settings: the rasterizer's parameters (the film size and camera come
    // from the scene); spp: samples per pixel per RasterizeScene; passes:
    // how many progressive passes they are split into (progress is reported
    // between passes and within them).
    GpuPathTracingSpectralRasterizer(const rtb200_render_settings& settings, unsigned int spp,
                                     unsigned int passes, int device = 0);

    void AttachToScene(const IScene* pScene) override;
    void DetachFromScene(const IScene* pScene) override;
    unsigned int PredictTimeToRasterizeScene(const IScene&, const ISampling2D&, unsigned int* pActualTime) const override;
    void RasterizeScene(const IScene& pScene, const Rect* pRect, IRasterizeSequence* pRasterSequence) const override;
    void RasterizeSceneAnimation(const IScene& pScene, const Scalar time_start, const Scalar time_end,
                                 const unsigned int num_frames, const bool do_fields, const bool invert_fields,
                                 const Rect* pRect, const unsigned int* specificFrame,
                                 IRasterizeSequence* pRasterSequence) const override;

    // Status of the last RasterizeScene (an RTB200_* code) and its message.
    int LastStatus() const { return last_status; }
    const std::string& LastMessage() const { return last_message; }
    // What the last extraction refused (empty when the whole scene was read).
    const std::vector<std::string>& Refused() const { return refused; }

protected:
    virtual ~GpuPathTracingSpectralRasterizer();

private:
    rtb200_render_settings base;
    unsigned int spp, passes;
    int device;
    mutable rtb200_ctx* ctx = nullptr;
    mutable rtb200_scene* dev_scene = nullptr;
    mutable const IScene* dev_for = nullptr;
    mutable rtb200_render_settings job_settings{};
    mutable int last_status = RTB200_OK;
    mutable std::string last_message;
    mutable std::vector<std::string> refused;
};

}  // namespace Implementation
}  // namespace RISE
