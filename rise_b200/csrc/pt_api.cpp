// pt_api.cpp -- C ABI of the spectral path tracer: spectra, materials,
// luminaries, and progressive render jobs (include/rtb200.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "cie1931.h"
#include "core.h"
#include "ggx_tables.h"
#include "pathtrace.h"

namespace rtb200 {

namespace {

const float kCieY[RTB200_CIE_COUNT] = {RTB200_CIE_YBAR};

// ColorUtils::CIE_Y_Integral (src/Library/Utilities/Color/ColorUtils.cpp:327-348):
// trapezoid sum of y-bar over whole 5 nm cells between the clamped bounds.
double CieYIntegral(double a, double b)
{
    const double lo = a < 380.0 ? 380.0 : a;
    const double hi = b > 780.0 ? 780.0 : b;
    if (hi <= lo) return 0.0;
    const int first = (int)((lo - 380.0) / 5.0);
    const int last = (int)((hi - 380.0) / 5.0);
    double sum = 0.0;
    for (int i = first; i < last; ++i) sum += 0.5 * ((double)kCieY[i] + (double)kCieY[i + 1]) * 5.0;
    return sum;
}

template <class T>
int Upload(rtb200_ctx* ctx, T** dst, const std::vector<T>& src, size_t& total)
{
    *dst = nullptr;
    if (src.empty()) return RTB200_OK;
    void* p = nullptr;
    int rc = DevAlloc(ctx, &p, src.size() * sizeof(T));
    if (rc) return rc;
    if (cudaMemcpy(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
        DevFree(ctx, p, src.size() * sizeof(T));
        return CudaCheck(ctx, cudaGetLastError(), "shading upload");
    }
    total += src.size() * sizeof(T);
    *dst = (T*)p;
    return RTB200_OK;
}

}  // namespace

int UploadShading(rtb200_scene* s)
{
    rtb200_ctx* ctx = s->ctx;
    if (s->materials.empty()) return RTB200_OK;  // ray casting only
    const size_t nm = s->materials.size();
    // GGX conductors: tabulate F_avg(lambda) on the 5 nm grid as an extra
    // spectrum, and make sure the device holds the E_ss / E_avg tables.
    for (PtMaterial& m : s->materials) {
        if (m.type != kMatGGX) continue;
        std::vector<float> favg(RTB200_CIE_COUNT);
        for (int k = 0; k < RTB200_CIE_COUNT; ++k) {
            const double eta = m.eta >= 0 ? s->spectra[(size_t)m.eta * RTB200_CIE_COUNT + k] : m.ior;
            const double kap = m.kappa >= 0 ? s->spectra[(size_t)m.kappa * RTB200_CIE_COUNT + k] : 0.0;
            favg[k] = (float)ConductorFresnelAvg(1.0, eta, kap);
        }
        m.pad = (int)(s->spectra.size() / RTB200_CIE_COUNT);
        s->spectra.insert(s->spectra.end(), favg.begin(), favg.end());
    }
    {
        const GgxTables& gt = GetGgxTables();
        const cudaError_t e = PtSetGgxTables(gt.ess, gt.eavg);
        if (e != cudaSuccess) return CudaCheck(ctx, e, "GGX tables");
    }
    for (const auto& mesh : s->meshes)
        if (mesh.material < 0 || (size_t)mesh.material >= nm)
            return SetError(ctx, RTB200_E_INVALID, "mesh material id out of range");
    // Luminaries: one per mesh whose material emits.
    s->lights.clear();
    s->light_tris.clear();
    std::vector<int> meshLight(s->meshes.size(), -1);
    std::vector<double> weight;
    for (size_t mi = 0; mi < s->meshes.size(); ++mi) {
        const auto& mesh = s->meshes[mi];
        const PtMaterial& mat = s->materials[mesh.material];
        if (mat.emit < 0 || mesh.count <= 0) continue;
        PtLight L{};
        L.first = (int)s->light_tris.size();
        L.count = (int)mesh.count;
        L.emit = mat.emit;
        double area = 0.0;
        std::vector<double> cum;
        for (int64_t t = mesh.first; t < mesh.first + mesh.count; ++t) {
            const float* v = &s->tri9[9 * (size_t)t];
            PtLightTri lt{};
            for (int k = 0; k < 3; ++k) { lt.v0[k] = v[k]; lt.e1[k] = v[3 + k] - v[k]; lt.e2[k] = v[6 + k] - v[k]; }
            const double cx = (double)lt.e1[1] * lt.e2[2] - (double)lt.e1[2] * lt.e2[1];
            const double cy = (double)lt.e1[2] * lt.e2[0] - (double)lt.e1[0] * lt.e2[2];
            const double cz = (double)lt.e1[0] * lt.e2[1] - (double)lt.e1[1] * lt.e2[0];
            area += 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
            cum.push_back(area);
            s->light_tris.push_back(lt);
        }
        if (!(area > 0.0)) { s->light_tris.resize(L.first); continue; }
        for (size_t k = 0; k < cum.size(); ++k) s->light_tris[L.first + k].cdf = (float)(cum[k] / area);
        s->light_tris[L.first + cum.size() - 1].cdf = 1.0f;
        L.area = (float)area;
        // Selection weight: emitted power, area x mean radiance over 380..780 nm.
        double mean = 0.0;
        for (int k = 0; k < RTB200_CIE_COUNT; ++k) mean += s->spectra[(size_t)mat.emit * RTB200_CIE_COUNT + k];
        mean /= RTB200_CIE_COUNT;
        weight.push_back(area * std::max(mean, 1e-12));
        meshLight[mi] = (int)s->lights.size();
        s->lights.push_back(L);
    }
    double wsum = 0.0;
    for (double w : weight) wsum += w;
    for (size_t i = 0; i < s->lights.size(); ++i) s->lights[i].pdf = (float)(weight[i] / wsum);
    // Per-triangle attributes in leaf order.
    const size_t ntri = s->tri_material.size();
    std::vector<int> triMesh(ntri);
    for (size_t mi = 0; mi < s->meshes.size(); ++mi)
        for (int64_t t = s->meshes[mi].first; t < s->meshes[mi].first + s->meshes[mi].count; ++t) triMesh[t] = (int)mi;
    std::vector<PtTriAttr> attr(ntri);
    for (size_t slot = 0; slot < ntri; ++slot) {
        const int mi = triMesh[s->bvh.prims[slot]];
        const auto& mesh = s->meshes[mi];
        attr[slot].mat = (mesh.material & kAttrMatMask) | (mesh.double_sided ? kAttrDoubleSided : 0);
        attr[slot].light = meshLight[mi];
    }
    size_t total = 0;
    int rc = Upload(ctx, &s->d_attr, attr, total);
    if (!rc) rc = Upload(ctx, &s->d_mats, s->materials, total);
    if (!rc) rc = Upload(ctx, &s->d_spectra, s->spectra, total);
    if (!rc) rc = Upload(ctx, &s->d_lights, s->lights, total);
    if (!rc) rc = Upload(ctx, &s->d_light_tris, s->light_tris, total);
    s->shade_bytes = total;
    if (rc) FreeShading(s);
    return rc;
}

void FreeShading(rtb200_scene* s)
{
    rtb200_ctx* ctx = s->ctx;
    DevFree(ctx, s->d_attr, s->tri_material.size() * sizeof(PtTriAttr));
    DevFree(ctx, s->d_mats, s->materials.size() * sizeof(PtMaterial));
    DevFree(ctx, s->d_spectra, s->spectra.size() * sizeof(float));
    DevFree(ctx, s->d_lights, s->lights.size() * sizeof(PtLight));
    DevFree(ctx, s->d_light_tris, s->light_tris.size() * sizeof(PtLightTri));
    s->d_attr = nullptr;
    s->d_mats = nullptr;
    s->d_spectra = nullptr;
    s->d_lights = nullptr;
    s->d_light_tris = nullptr;
    s->shade_bytes = 0;
}

}  // namespace rtb200

using namespace rtb200;

struct rtb200_job {
    rtb200_scene* scene = nullptr;
    rtb200_render_settings rs{};
    PtLaunch L{};
    int capacity = 0;
    int npix = 0;
    void* buf = nullptr;
    size_t bytes = 0;
    int* d_iota = nullptr;
    long long spp_done = 0;
    long long samples = 0;
    double seconds = 0.0;
    int* h_cnt = nullptr;                 // pinned: counters snapshot
    unsigned long long* h_u64 = nullptr;  // pinned: sample counter, stats
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

namespace {

size_t Align(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

int rtb200_scene_add_spectrum(rtb200_scene* s, const float* values, int32_t* id_out)
{
    if (!s || !values || !id_out) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    for (int k = 0; k < RTB200_CIE_COUNT; ++k)
        if (!std::isfinite(values[k]) || values[k] < 0.0f)
            return SetError(s->ctx, RTB200_E_INVALID, "spectrum values must be finite and non-negative");
    *id_out = (int32_t)(s->spectra.size() / RTB200_CIE_COUNT);
    s->spectra.insert(s->spectra.end(), values, values + RTB200_CIE_COUNT);
    return RTB200_OK;
}

int rtb200_scene_add_material(rtb200_scene* s, const rtb200_material* m, int32_t* id_out)
{
    if (!s || !m || !id_out) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    const int nspec = (int)(s->spectra.size() / RTB200_CIE_COUNT);
    auto okSpec = [&](int id) { return id >= -1 && id < nspec; };
    if (m->type < RTB200_MAT_LAMBERTIAN || m->type > RTB200_MAT_DIELECTRIC || !okSpec(m->reflectance) ||
        !okSpec(m->emission) || !okSpec(m->eta) || !okSpec(m->kappa))
        return SetError(s->ctx, RTB200_E_INVALID, "bad material");
    PtMaterial pm{};
    pm.type = m->type;
    pm.refl = m->reflectance;
    pm.emit = m->emission;
    pm.eta = m->eta;
    pm.kappa = m->kappa;
    pm.alpha = m->alpha;
    pm.ior = m->ior;
    pm.pad = -1;   // conductor Fresnel average spectrum, built at commit
    *id_out = (int32_t)s->materials.size();
    s->materials.push_back(pm);
    return RTB200_OK;
}

int rtb200_scene_set_environment(rtb200_scene* s, int32_t spectrum, int32_t visible)
{
    if (!s) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    if (spectrum < -1 || spectrum >= (int32_t)(s->spectra.size() / RTB200_CIE_COUNT))
        return SetError(s->ctx, RTB200_E_INVALID, "bad environment spectrum");
    s->env = spectrum;
    s->env_visible = visible ? 1 : 0;
    return RTB200_OK;
}

int rtb200_job_create(rtb200_scene* s, const rtb200_render_settings* rs, rtb200_job** out)
{
    if (!s || !rs || !out) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    *out = nullptr;
    if (!s->committed || s->materials.empty())
        return SetError(ctx, RTB200_E_INVALID, "scene must be committed with materials");
    if (rs->width <= 0 || rs->height <= 0 || (int64_t)rs->width * rs->height > (1ll << 28) || rs->max_depth < 1 ||
        rs->max_depth > 255 || !(rs->lambda_max > rs->lambda_min) || rs->lambda_min < 380.0f ||
        rs->lambda_max > 780.0f || !(rs->fov_deg > 0.0f && rs->fov_deg < 180.0f))
        return SetError(ctx, RTB200_E_INVALID, "bad render settings");
    cudaSetDevice(ctx->device);
    rtb200_job* j = new (std::nothrow) rtb200_job();
    if (!j) return SetError(ctx, RTB200_E_OOM, "host allocation failed");
    j->scene = s;
    j->rs = *rs;
    j->npix = rs->width * rs->height;
    int cap = rs->max_paths > 0 ? rs->max_paths : std::min(std::max(j->npix * 8, 65536), 1 << 21);
    cap = (cap + 31) & ~31;
    j->capacity = cap;
    // One device allocation carved into the path pool, queues, film, counters.
    const size_t c = (size_t)cap, np = (size_t)j->npix;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t at = off; off += Align(bytes); return at; };
    const size_t oRo = take(16 * c), oRd = take(16 * c), oHit = take(16 * c), oThr = take(16 * c), oL = take(16 * c),
                 oAux = take(16 * c), oMeta = take(16 * c);
    const size_t oQa = take(4 * c), oQan = take(4 * c), oQf = take(4 * c), oQfn = take(4 * c), oIota = take(4 * c);
    const size_t oSh = take(sizeof(ShadowEntry) * 8 * c);   // up to 4 light + 4 sky samples
    const size_t oPass = take(12 * np), oSum = take(12 * np), oComp = take(12 * np);
    const size_t oCnt = take(4 * kCntCount), oU64 = take(8 * 8), oErr = take(4);
    int rc = DevAlloc(ctx, &j->buf, off);
    if (rc) { delete j; return rc; }
    j->bytes = off;
    char* b = (char*)j->buf;
    cudaMemset(b, 0, off);
    PtLaunch& L = j->L;
    L.sms = ctx->num_sms;
    L.scene = PtScene{s->d_nodes, s->layout, s->d_tris, (int)s->tri_material.size(), s->d_attr, s->d_mats,
                      s->d_spectra, s->d_lights, s->d_light_tris};
    L.paths = PtPaths{(float4*)(b + oRo), (float4*)(b + oRd), (float4*)(b + oHit), (float4*)(b + oThr),
                      (float4*)(b + oL), (float4*)(b + oAux), (uint4*)(b + oMeta)};
    unsigned long long* u64 = (unsigned long long*)(b + oU64);
    L.queues = PtQueues{(int*)(b + oQa), (int*)(b + oQan), (int*)(b + oQf), (int*)(b + oQfn),
                        (ShadowEntry*)(b + oSh), (int*)(b + oCnt), u64, u64 + 1, (unsigned*)(b + oErr)};
    L.film = PtFilm{(float*)(b + oPass), (float*)(b + oSum), (float*)(b + oComp)};
    j->d_iota = (int*)(b + oIota);
    {
        std::vector<int> iota(c);
        for (size_t i = 0; i < c; ++i) iota[i] = (int)i;
        cudaMemcpy(j->d_iota, iota.data(), 4 * c, cudaMemcpyHostToDevice);
    }
    // Camera frame (pinhole; vertical field of view).
    PtCamera& cam = L.params.cam;
    const float* P = rs->cam_pos;
    double f[3] = {rs->cam_look[0] - P[0], rs->cam_look[1] - P[1], rs->cam_look[2] - P[2]};
    double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (double& x : f) x /= fl;
    const double* u = nullptr;
    double up[3] = {rs->cam_up[0], rs->cam_up[1], rs->cam_up[2]};
    u = up;
    double r[3] = {f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0]};
    double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (!(rl > 0.0) || !(fl > 0.0)) {
        DevFree(ctx, j->buf, j->bytes);
        delete j;
        return SetError(ctx, RTB200_E_INVALID, "degenerate camera frame");
    }
    for (double& x : r) x /= rl;
    double uu[3] = {r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]};
    const double th = std::tan(0.5 * rs->fov_deg * 3.14159265358979323846 / 180.0);
    const double aspect = (double)rs->width / (double)rs->height;
    for (int k = 0; k < 3; ++k) {
        cam.pos[k] = P[k];
        cam.fwd[k] = (float)f[k];
        cam.right[k] = (float)(r[k] * th * aspect);
        cam.up[k] = (float)(uu[k] * th);
    }
    cam.width = rs->width;
    cam.height = rs->height;
    PtSettings& st = L.params.set;
    st.lmin = rs->lambda_min;
    st.lmax = rs->lambda_max;
    const double ky = CieYIntegral(rs->lambda_min, rs->lambda_max);
    st.ynorm = ky > 0.0 ? (float)((rs->lambda_max - rs->lambda_min) / ky) : 0.0f;
    st.max_depth = rs->max_depth;
    st.rr_min_depth = rs->rr_min_depth;
    st.rr_threshold = rs->rr_threshold;
    st.nee_per_lambda = rs->nee_per_lambda ? 1 : 0;
    st.seed = rs->seed;
    st.env = s->env;
    st.env_visible = s->env_visible;
    st.n_lights = (int)s->lights.size();
    st.n_spectra = (int)(s->spectra.size() / RTB200_CIE_COUNT);
    L.params.npix = j->npix;
    L.params.capacity = cap;
    if (cudaMallocHost(&j->h_cnt, 4 * kCntCount) != cudaSuccess || cudaMallocHost(&j->h_u64, 8 * 8) != cudaSuccess ||
        cudaEventCreate(&j->e0) != cudaSuccess || cudaEventCreate(&j->e1) != cudaSuccess) {
        cudaGetLastError();
        if (j->h_cnt) cudaFreeHost(j->h_cnt);
        if (j->h_u64) cudaFreeHost(j->h_u64);
        DevFree(ctx, j->buf, j->bytes);
        delete j;
        return SetError(ctx, RTB200_E_OOM, "pinned host allocation failed");
    }
    *out = j;
    return RTB200_OK;
}

int rtb200_job_render(rtb200_job* j, int32_t spp)
{
    if (!j) return RTB200_E_INVALID;
    rtb200_ctx* ctx = j->scene->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (spp <= 0) return SetError(ctx, RTB200_E_INVALID, "spp must be positive");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    PtLaunch L = j->L;
    L.params.sample_begin = (unsigned long long)j->spp_done;
    L.params.total = (unsigned long long)j->npix * (unsigned long long)spp;
    // Every slot starts free; counters (except the statistics) and the
    // sample counter restart.
    cudaMemcpyAsync(L.queues.free_, j->d_iota, 4 * (size_t)j->capacity, cudaMemcpyDeviceToDevice, st);
    {
        int init[kCntCount] = {0};
        init[kCntFree] = j->capacity;
        // Keep the running statistics in slots kCntSegments / kCntShadowRays.
        cudaMemcpyAsync(j->h_cnt, L.queues.cnt, 4 * kCntCount, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        init[kCntSegments] = j->h_cnt[kCntSegments];
        init[kCntShadowRays] = j->h_cnt[kCntShadowRays];
        std::memcpy(j->h_cnt, init, sizeof(init));
        cudaMemcpyAsync(L.queues.cnt, j->h_cnt, 4 * kCntCount, cudaMemcpyHostToDevice, st);
    }
    cudaMemsetAsync(L.queues.sample_ctr, 0, 8, st);
    cudaEventRecord(j->e0, st);
    const int kBatch = 4;
    const long long kMaxIterations = 1ll << 20;
    long long it = 0;
    cudaError_t e = cudaSuccess;
    for (;;) {
        for (int k = 0; k < kBatch; ++k) {
            e = PtIteration(L, st);
            if (e != cudaSuccess) break;
            std::swap(L.queues.active, L.queues.active_next);
            std::swap(L.queues.free_, L.queues.free_next);
        }
        if (e != cudaSuccess) break;
        it += kBatch;
        cudaMemcpyAsync(j->h_cnt, L.queues.cnt, 4 * kCntCount, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(j->h_u64, L.queues.sample_ctr, 8, cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) break;
        if (j->h_cnt[kCntActive] == 0 && j->h_cnt[kCntFree] == 0 && j->h_u64[0] >= L.params.total) break;
        if (it > kMaxIterations) return SetError(ctx, RTB200_E_TIMEOUT, "render did not drain its path queues");
    }
    if (e == cudaSuccess) e = PtFold(L.film, j->npix, L.sms, st);
    if (e == cudaSuccess) e = cudaEventRecord(j->e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(j->e1);
    if (e != cudaSuccess) return CudaCheck(ctx, e, "render");
    unsigned err = 0;
    cudaMemcpy(&err, L.queues.err, 4, cudaMemcpyDeviceToHost);
    if (err) return SetError(ctx, RTB200_E_DEVICE, "device error word set (traversal stack overflow)");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, j->e0, j->e1);
    j->seconds += ms * 1e-3;
    j->spp_done += spp;
    j->samples += (long long)j->npix * spp;
    // Queue buffers may have been swapped an odd number of times.
    j->L.queues.active = L.queues.active;
    j->L.queues.active_next = L.queues.active_next;
    j->L.queues.free_ = L.queues.free_;
    j->L.queues.free_next = L.queues.free_next;
    return RTB200_OK;
}

int rtb200_job_read_film(rtb200_job* j, float* xyz)
{
    if (!j || !xyz) return RTB200_E_INVALID;
    rtb200_ctx* ctx = j->scene->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    const size_t n3 = 3 * (size_t)j->npix;
    std::vector<float> sum(n3), comp(n3);
    cudaError_t e = cudaMemcpy(sum.data(), j->L.film.sum, 4 * n3, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(comp.data(), j->L.film.comp, 4 * n3, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return CudaCheck(ctx, e, "film readback");
    const double inv = j->spp_done > 0 ? 1.0 / (double)j->spp_done : 0.0;
    for (size_t i = 0; i < n3; ++i) xyz[i] = (float)(((double)sum[i] - (double)comp[i]) * inv);
    return RTB200_OK;
}

int rtb200_job_stats(const rtb200_job* j, rtb200_stats* out)
{
    if (!j || !out) return RTB200_E_INVALID;
    int cnt[kCntCount];
    cudaMemcpy(cnt, j->L.queues.cnt, sizeof(cnt), cudaMemcpyDeviceToHost);
    out->spp = j->spp_done;
    out->samples = j->samples;
    out->segments = (unsigned)cnt[kCntSegments];
    out->shadow_rays = (unsigned)cnt[kCntShadowRays];
    out->seconds = j->seconds;
    return RTB200_OK;
}

int rtb200_job_destroy(rtb200_job* j)
{
    if (!j) return RTB200_E_INVALID;
    rtb200_ctx* ctx = j->scene->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    DevFree(ctx, j->buf, j->bytes);
    if (j->h_cnt) cudaFreeHost(j->h_cnt);
    if (j->h_u64) cudaFreeHost(j->h_u64);
    if (j->e0) cudaEventDestroy(j->e0);
    if (j->e1) cudaEventDestroy(j->e1);
    delete j;
    return RTB200_OK;
}

}  // extern "C"
