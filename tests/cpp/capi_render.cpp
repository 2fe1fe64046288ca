// capi_render.cpp -- a C++ host program on the rtb200 C ABI, the way a RISE
// build drives it from its rasterizer (IRasterizer::RasterizeScene ->
// PixelBasedRasterizerHelper's progressive passes): scene extraction into
// rtb200_scene_*, one rtb200_job, progressive rtb200_job_render passes, and
// the film read back for the rasterizer outputs.
//
// Usage: capi_render <scene.bin> <film.out>
//   scene.bin (little endian): "RTBS", int32 version 1,
//     int32 n_spectra, n_spectra x 81 float,
//     int32 n_materials, n_materials x rtb200_material,
//     int32 environment spectrum, int32 environment visible,
//     int32 n_meshes, per mesh: int64 n_tri, int32 material, int32 double
//       sided, n_tri x 9 float (v0, v1, v2),
//     rtb200_render_settings,
//     int32 n_passes, n_passes x int32 spp.
//   film.out: width * height * 3 float (mean XYZ per pixel, rows top to bottom).
// Prints one line "spp=<n> samples=<n> segments=<n> shadow_rays=<n>".
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rtb200.h"

namespace {

struct Reader {
    FILE* f;
    bool ok = true;
    template <class T>
    T get()
    {
        T v{};
        ok = ok && std::fread(&v, sizeof(T), 1, f) == 1;
        return v;
    }
    void bytes(void* p, size_t n) { ok = ok && std::fread(p, 1, n, f) == n; }
};

int Fail(rtb200_ctx* ctx, const char* what, int rc)
{
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, ctx ? rtb200_last_error(ctx) : "");
    return 1;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s scene.bin film.out\n", argv[0]);
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) { std::perror(argv[1]); return 1; }
    Reader r{in};
    char magic[4];
    r.bytes(magic, 4);
    if (!r.ok || std::memcmp(magic, "RTBS", 4) != 0 || r.get<int32_t>() != 1) {
        std::fprintf(stderr, "not a version-1 scene file\n");
        return 1;
    }
    rtb200_ctx* ctx = nullptr;
    int rc = rtb200_ctx_create(0, 0, &ctx);
    if (rc) return Fail(nullptr, "rtb200_ctx_create", rc);
    rtb200_scene* scene = nullptr;
    if ((rc = rtb200_scene_create(ctx, &scene))) return Fail(ctx, "rtb200_scene_create", rc);

    const int32_t n_spec = r.get<int32_t>();
    std::vector<float> spectrum(RTB200_SPECTRUM_SAMPLES);
    for (int32_t i = 0; i < n_spec && r.ok; ++i) {
        r.bytes(spectrum.data(), sizeof(float) * spectrum.size());
        int32_t id;
        if ((rc = rtb200_scene_add_spectrum(scene, spectrum.data(), &id))) return Fail(ctx, "add_spectrum", rc);
    }
    const int32_t n_mat = r.get<int32_t>();
    for (int32_t i = 0; i < n_mat && r.ok; ++i) {
        const rtb200_material m = r.get<rtb200_material>();
        int32_t id;
        if ((rc = rtb200_scene_add_material(scene, &m, &id))) return Fail(ctx, "add_material", rc);
    }
    const int32_t env = r.get<int32_t>(), env_visible = r.get<int32_t>();
    if ((rc = rtb200_scene_set_environment(scene, env, env_visible))) return Fail(ctx, "set_environment", rc);
    const int32_t n_mesh = r.get<int32_t>();
    for (int32_t i = 0; i < n_mesh && r.ok; ++i) {
        const int64_t n_tri = r.get<int64_t>();
        const int32_t material = r.get<int32_t>(), double_sided = r.get<int32_t>();
        std::vector<float> xyz(9 * (size_t)n_tri);
        r.bytes(xyz.data(), sizeof(float) * xyz.size());
        std::vector<uint32_t> tri(3 * (size_t)n_tri);
        for (size_t k = 0; k < tri.size(); ++k) tri[k] = (uint32_t)k;
        if ((rc = rtb200_scene_add_mesh(scene, xyz.data(), 3 * n_tri, tri.data(), n_tri, material, double_sided)))
            return Fail(ctx, "add_mesh", rc);
    }
    const rtb200_render_settings settings = r.get<rtb200_render_settings>();
    const int32_t n_pass = r.get<int32_t>();
    std::vector<int32_t> passes(n_pass > 0 ? n_pass : 0);
    for (auto& p : passes) p = r.get<int32_t>();
    std::fclose(in);
    if (!r.ok) { std::fprintf(stderr, "truncated scene file\n"); return 1; }

    if ((rc = rtb200_scene_commit(scene, RTB200_BVH_F32))) return Fail(ctx, "rtb200_scene_commit", rc);
    rtb200_job* job = nullptr;
    if ((rc = rtb200_job_create(scene, &settings, &job))) return Fail(ctx, "rtb200_job_create", rc);
    for (int32_t spp : passes)
        if ((rc = rtb200_job_render(job, spp))) return Fail(ctx, "rtb200_job_render", rc);
    std::vector<float> film(3 * (size_t)settings.width * settings.height);
    if ((rc = rtb200_job_read_film(job, film.data()))) return Fail(ctx, "rtb200_job_read_film", rc);
    rtb200_stats st;
    if ((rc = rtb200_job_stats(job, &st))) return Fail(ctx, "rtb200_job_stats", rc);
    FILE* out = std::fopen(argv[2], "wb");
    if (!out || std::fwrite(film.data(), sizeof(float), film.size(), out) != film.size()) {
        std::perror(argv[2]);
        return 1;
    }
    std::fclose(out);
    std::printf("spp=%lld samples=%lld segments=%lld shadow_rays=%lld\n", (long long)st.spp, (long long)st.samples,
                (long long)st.segments, (long long)st.shadow_rays);
    rtb200_job_destroy(job);
    rtb200_scene_destroy(scene);
    rtb200_ctx_destroy(ctx);
    return 0;
}
