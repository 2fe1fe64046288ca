// rise_adapter_check.cpp -- TEST PROGRAM for the RISE-side adapter
// (rise_b200/adapter/): loads a .RISEscene with the reference renderer's own
// job and parser (oracle/_ref/librise_ref.so), then
//
//   rise_adapter_check extract scene.RISEscene out_prefix
//       reads the parsed IScene through rtb200_rise::ExtractScene and writes
//       out_prefix.json (spectra, materials, meshes, environment, camera,
//       film, refusals) and out_prefix.xyz (every mesh's world-space corner
//       positions, float32) for comparison with this package's scene ingest;
//
//   rise_adapter_check render scene.RISEscene settings.bin spp passes out.rgb
//       swaps the job's rasterizer for GpuPathTracingSpectralRasterizer
//       (settings.bin: an rtb200_render_settings; film and camera come from
//       the scene), rasterizes through the job, and writes the image the
//       rasterizer hands its outputs (width x height x 3 float32 linear
//       Rec.709, rows from the top) to out.rgb; prints "ok <status>".
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "Interfaces/IJobPriv.h"
#include "Interfaces/IRasterImage.h"
#include "Interfaces/IRasterizerOutput.h"
#include "Interfaces/IScenePriv.h"
#include "Utilities/MediaPathLocator.h"
#include "Utilities/Reference.h"
#include "gpu_rasterizer.h"
#include "rise_extract.h"

using namespace RISE;
using namespace RISE::Implementation;

namespace {

class Capture : public virtual IRasterizerOutput, public virtual Reference
{
public:
    std::vector<float> rgb;
    unsigned int width = 0, height = 0;

protected:
    virtual ~Capture() {}

public:
    void OutputIntermediateImage(const IRasterImage&, const Rect*) override {}
    void OutputImage(const IRasterImage& img, const Rect*, const unsigned int) override
    {
        width = img.GetWidth();
        height = img.GetHeight();
        rgb.resize((size_t)width * height * 3);
        for (unsigned int y = 0; y < height; ++y)
            for (unsigned int x = 0; x < width; ++x) {
                const RISEColor c = img.GetPEL(x, y);
                float* o = &rgb[3 * ((size_t)y * width + x)];
                o[0] = (float)c.base.r;
                o[1] = (float)c.base.g;
                o[2] = (float)c.base.b;
            }
    }
};

IJobPriv* Load(const char* path)
{
    std::string dir(path);
    const size_t cut = dir.find_last_of('/');
    dir = cut == std::string::npos ? std::string("./") : dir.substr(0, cut + 1);
    GlobalMediaPathLocator().AddPath(dir.c_str());
    IJobPriv* job = nullptr;
    if (!RISE_CreateJobPriv(&job) || !job) return nullptr;
    if (!job->LoadAsciiSceneViaCst(path)) {
        safe_release(job);
        return nullptr;
    }
    return job;
}

void Floats(FILE* f, const float* v, size_t n)
{
    std::fputc('[', f);
    for (size_t i = 0; i < n; ++i) std::fprintf(f, "%s%.9g", i ? ", " : "", v[i]);
    std::fputc(']', f);
}

int Extract(const char* scene_path, const std::string& prefix)
{
    IJobPriv* job = Load(scene_path);
    if (!job) return 2;
    rtb200_rise::Scene ex;
    rtb200_rise::ExtractScene(*job->GetScene(), ex);
    FILE* f = std::fopen((prefix + ".json").c_str(), "w");
    if (!f) return 3;
    std::fprintf(f, "{\"width\": %d, \"height\": %d, \"fov_deg\": %.9g, \"cam_pos\": ", ex.width, ex.height, ex.fov_deg);
    Floats(f, ex.cam_pos, 3);
    std::fprintf(f, ", \"cam_look\": ");
    Floats(f, ex.cam_look, 3);
    std::fprintf(f, ", \"cam_up\": ");
    Floats(f, ex.cam_up, 3);
    std::fprintf(f, ",\n \"spectra\": [");
    for (size_t i = 0; i < ex.spectra.size(); ++i) {
        const rtb200_rise::Spectrum& s = ex.spectra[i];
        std::fprintf(f, "%s{\"kind\": %d, \"begin\": %.9g, \"end\": %.9g, \"coeffs\": [%.17g, %.17g, %.17g, %.17g], \"amps\": ",
                     i ? ",\n  " : "", s.kind, s.begin, s.end, s.coeffs[0], s.coeffs[1], s.coeffs[2], s.coeffs[3]);
        Floats(f, s.amps.data(), s.amps.size());
        std::fputc('}', f);
    }
    std::fprintf(f, "],\n \"materials\": [");
    for (size_t i = 0; i < ex.materials.size(); ++i) {
        const rtb200_material& m = ex.materials[i];
        std::fprintf(f, "%s[%d, %d, %d, %d, %d, %.9g, %.9g]", i ? ", " : "", m.type, m.reflectance, m.emission, m.eta,
                     m.kappa, m.alpha, m.ior);
    }
    std::fprintf(f, "],\n \"meshes\": [");
    for (size_t i = 0; i < ex.meshes.size(); ++i) {
        const rtb200_rise::Mesh& m = ex.meshes[i];
        std::fprintf(f, "%s{\"triangles\": %zu, \"material\": %d, \"double_sided\": %d, \"normals\": %d}",
                     i ? ", " : "", m.xyz.size() / 9, m.material, m.double_sided, m.nrm.empty() ? 0 : 1);
    }
    std::fprintf(f, "],\n \"env_spectrum\": %d, \"env_visible\": %d, \"env_image\": [%d, %d, %.9g], \"env_rot\": ",
                 ex.env_spectrum, ex.env_visible, ex.env_image.width, ex.env_image.height, ex.env_image.scale);
    Floats(f, ex.env_image.rot, 9);
    std::fprintf(f, ",\n \"refused\": [");
    for (size_t i = 0; i < ex.refused.size(); ++i) std::fprintf(f, "%s\"%s\"", i ? ", " : "", ex.refused[i].c_str());
    std::fprintf(f, "]}\n");
    std::fclose(f);
    f = std::fopen((prefix + ".xyz").c_str(), "wb");
    if (!f) return 3;
    for (const rtb200_rise::Mesh& m : ex.meshes) std::fwrite(m.xyz.data(), 4, m.xyz.size(), f);
    std::fclose(f);
    if (ex.env_image.width > 0) {
        f = std::fopen((prefix + ".env").c_str(), "wb");
        if (!f) return 3;
        std::fwrite(ex.env_image.rgb.data(), 4, ex.env_image.rgb.size(), f);
        std::fclose(f);
    }
    safe_release(job);
    std::printf("ok %zu %zu\n", ex.meshes.size(), ex.refused.size());
    return 0;
}

int Render(const char* scene_path, const char* settings_path, unsigned int spp, unsigned int passes,
           const char* out_path)
{
    rtb200_render_settings rs;
    FILE* f = std::fopen(settings_path, "rb");
    if (!f || std::fread(&rs, sizeof(rs), 1, f) != 1) return 2;
    std::fclose(f);
    IJobPriv* job = Load(scene_path);
    if (!job) return 2;
    job->RemoveRasterizerOutputs();
    GpuPathTracingSpectralRasterizer* rast = new GpuPathTracingSpectralRasterizer(rs, spp, passes, 0);
    Capture* cap = new Capture();
    rast->AddRasterizerOutput(cap);
    // Rasterize the parsed scene through the IRasterizer interface, as
    // Job::Rasterize does with the rasterizer it holds.
    IRasterizer* as_interface = rast;
    as_interface->RasterizeScene(*job->GetScene(), nullptr, nullptr);
    int rc = 0;
    if (rast->LastStatus() != RTB200_OK || cap->rgb.empty()) {
        std::printf("error %d %s\n", rast->LastStatus(), rast->LastMessage().c_str());
        rc = 4;
    } else {
        f = std::fopen(out_path, "wb");
        std::fwrite(cap->rgb.data(), 4, cap->rgb.size(), f);
        std::fclose(f);
        std::printf("ok %d %u %u\n", rast->LastStatus(), cap->width, cap->height);
    }
    safe_release(cap);
    safe_release(rast);
    safe_release(job);
    return rc;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc == 4 && !std::strcmp(argv[1], "extract")) return Extract(argv[2], argv[3]);
    if (argc == 7 && !std::strcmp(argv[1], "render"))
        return Render(argv[2], argv[3], (unsigned)std::atoi(argv[4]), (unsigned)std::atoi(argv[5]), argv[6]);
    std::fprintf(stderr, "usage: rise_adapter_check extract scene prefix | render scene settings spp passes out\n");
    return 1;
}
