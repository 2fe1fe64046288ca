// engine.cpp -- render jobs and the shared wavefront engine (include/rtb200.h).
//
// A job is one image: its scene, camera, settings and film (compensated
// running sums plus this request's accumulator).  An engine owns a pool of
// path slots, the ray / shadow-ray queues and a table of up to kMaxJobs job
// descriptors.  Any number of jobs -- of different scenes and resolutions --
// share one engine: every wavefront iteration regenerates free slots with
// camera samples of whichever jobs still have samples to hand out, so the
// jobs' work overlaps on the device (batched rendering, and continuous
// batching when jobs are submitted while others are in flight).  A job
// rendered alone (rtb200_job_render) uses a private engine.
//
// The reference renders one image at a time on a CPU thread pool
// (PixelBasedRasterizerHelper::RasterizeScene, progressive passes at
// Rendering/PixelBasedRasterizerHelper.cpp:1159-1293); a job's request of N
// samples per pixel corresponds to one progressive pass of N samples.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "cie1931.h"
#include "core.h"
#include "pathtrace.h"

using namespace rtb200;

namespace {

constexpr int kMaxJobs = kPtMaxJobs;
constexpr long long kWideSpp = 4096;   // samples per pixel kept in the compensated FP32 film
// Requests of at least this many samples per pixel fold their FP32 pass film
// into the running sum after every engine step, so no FP32 atomic sum spans
// more than one step's worth of samples.
constexpr long long kFoldEverySpp = 64;
constexpr int kGraphIters = 2;   // iterations per captured graph (even: queue pointers return)

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

size_t Align(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct rtb200_job {
    rtb200_scene* scene = nullptr;
    rtb200_render_settings rs{};
    PtCamera cam{};
    PtSettings set{};
    int npix = 0;
    int channels = 3;                  // floats per film pixel: XYZ (+ weight when splatted)
    int film_n = 0;                    // channels * npix
    void* film_buf = nullptr;
    size_t film_bytes = 0;
    float* pass = nullptr;
    float* sum = nullptr;
    float* comp = nullptr;
    double* wide = nullptr;            // FP64 running sum once past kWideSpp samples per pixel
    // Adaptive sampling: lists of the pixels still sampled (current and
    // next), samples per pixel, per-pixel sums of Y and Y^2, list length.
    bool adaptive = false;
    void* adapt_buf = nullptr;
    size_t adapt_bytes = 0;
    unsigned* px_list[2] = {nullptr, nullptr};
    unsigned* counts = nullptr;
    double* lum = nullptr;
    int* d_n = nullptr;
    int cur = 0;
    int n_active = 0;                  // pixels the next request samples
    int submitted_px = 0;              // pixels the request in flight samples
    long long spp_done = 0;
    int spectral = 1;                  // paths per pixel sample (spectral samples)
    rtb200_progress_fn progress = nullptr;   // rtb200_job_set_progress
    void* progress_user = nullptr;
    long long samples = 0;
    double seconds = 0.0;
    long long segments = 0, shadow_rays = 0;
    rtb200_engine* engine = nullptr;   // engine the job is submitted to
    int entry = -1;
    long long pending_spp = 0;
    rtb200_engine* own = nullptr;      // private engine of rtb200_job_render
};

struct rtb200_engine {
    rtb200_ctx* ctx = nullptr;
    int capacity = 0;
    int poll = 4;                          // iterations between host polls in EngineRender
    int layout = -1;
    void* buf = nullptr;
    size_t bytes = 0;
    PtPaths paths{};
    PtQueues queues{};
    int* d_iota = nullptr;
    PtJobDev* d_table = nullptr;
    int* d_ids = nullptr;
    unsigned long long* d_ctr = nullptr;   // [kMaxJobs] issued, [kMaxJobs] done
    PtJobDev* h_table = nullptr;           // pinned
    int* h_ids = nullptr;                  // pinned
    int* h_cnt = nullptr;                  // pinned
    unsigned long long* h_ctr = nullptr;   // pinned
    rtb200_job* owner[kMaxJobs] = {};
    unsigned long long total[kMaxJobs] = {};
    std::vector<int> active;
    std::vector<int> changed;              // table entries to upload before the next step
    bool dirty = true;
    bool fresh = true;
    int iter = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool ggraph = false;                   // gexec holds a capture for the fields below
    int glayout = -1;
    bool gspill = false;
    const rtb200_scene* gscene = nullptr;  // the shared scene, or null when jobs differ
    bool gclassify = false;
    bool genv_image = false;
    int gshade_class = -1;
    long long seg_seen = 0, shadow_seen = 0;
};

namespace {

PtLaunch MakeLaunch(const rtb200_engine* e)
{
    PtLaunch L;
    L.jobs = e->d_table;
    L.ids = e->d_ids;
    L.layout = e->layout;
    L.spill = false;
    L.uniform = !e->active.empty();
    L.classify = false;
    L.env_image = false;
    L.shade_class = e->active.empty() ? -1 : e->owner[e->active[0]]->scene->shade_class;
    for (int k : e->active) {
        L.env_image |= e->owner[k]->scene->d_env != nullptr;
        L.spill |= e->owner[k]->scene->stack_bound > kTraceStackShared;
        L.classify |= e->owner[k]->scene->mixed_shading;
        L.uniform &= e->owner[k]->scene == e->owner[e->active[0]]->scene;
        if (e->owner[k]->scene->shade_class != L.shade_class) L.shade_class = -1;
    }
    if (L.classify) L.shade_class = -1;
    L.scene = L.uniform ? e->h_table[e->active[0]].scene : PtScene{};
    L.paths = e->paths;
    L.queues = e->queues;
    L.sms = e->ctx->num_sms;
    return L;
}

void DropGraph(rtb200_engine* e)
{
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    e->gexec = nullptr;
    e->ggraph = false;
}

int EngineCreate(rtb200_ctx* ctx, int capacity, rtb200_engine** out)
{
    *out = nullptr;
    if (capacity <= 0) capacity = 1 << 21;
    capacity = (capacity + 31) & ~31;
    rtb200_engine* e = new (std::nothrow) rtb200_engine();
    if (!e) return SetError(ctx, RTB200_E_OOM, "host allocation failed");
    e->ctx = ctx;
    e->capacity = capacity;
    const size_t c = (size_t)capacity;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t at = off; off += Align(bytes); return at; };
    const size_t oRo = take(16 * c), oRd = take(16 * c), oHit = take(16 * c), oThr = take(16 * c), oL = take(16 * c),
                 oAux = take(16 * c), oMeta = take(16 * c), oMed = take(16 * c);
    const size_t oQa = take(4 * c), oQan = take(4 * c), oQf = take(4 * c), oQfn = take(4 * c), oIota = take(4 * c);
    const size_t oSh = take(sizeof(ShadowEntry) * 8 * c);   // up to 4 light + 4 sky samples per path
    const size_t oTab = take(sizeof(PtJobDev) * kMaxJobs), oIds = take(4 * kMaxJobs),
                 oCtr = take(8 * 2 * kMaxJobs);
    const size_t oCnt = take(4 * kCntCount), oTr = take(8 * 2), oSmp = take(8), oErr = take(4),
                 oAsg = take(sizeof(PtAssign) * kMaxJobs), oShd = take(4 * c * kShadeClasses);
    int rc = DevAlloc(ctx, &e->buf, off);
    if (rc) { delete e; return rc; }
    e->bytes = off;
    char* b = (char*)e->buf;
    cudaMemset(b, 0, off);
    e->paths = PtPaths{(float4*)(b + oRo), (float4*)(b + oRd), (float4*)(b + oHit), (float4*)(b + oThr),
                       (float4*)(b + oL), (float4*)(b + oAux), (uint4*)(b + oMeta), (int4*)(b + oMed)};
    e->queues = PtQueues{(int*)(b + oQa), (int*)(b + oQan), (int*)(b + oQf), (int*)(b + oQfn),
                         (ShadowEntry*)(b + oSh), (int*)(b + oCnt), (unsigned long long*)(b + oSmp),
                         (unsigned long long*)(b + oTr), (unsigned*)(b + oErr), (PtAssign*)(b + oAsg),
                         (int*)(b + oShd), capacity};
    e->d_iota = (int*)(b + oIota);
    e->d_table = (PtJobDev*)(b + oTab);
    e->d_ids = (int*)(b + oIds);
    e->d_ctr = (unsigned long long*)(b + oCtr);
    {
        std::vector<int> iota(c);
        for (size_t i = 0; i < c; ++i) iota[i] = (int)i;
        cudaMemcpy(e->d_iota, iota.data(), 4 * c, cudaMemcpyHostToDevice);
    }
    if (cudaMallocHost(&e->h_table, sizeof(PtJobDev) * kMaxJobs) != cudaSuccess ||
        cudaMallocHost(&e->h_ids, 4 * (kMaxJobs + 1)) != cudaSuccess ||
        cudaMallocHost(&e->h_cnt, 4 * kCntCount) != cudaSuccess ||
        cudaMallocHost(&e->h_ctr, 8 * 2 * kMaxJobs) != cudaSuccess || cudaEventCreate(&e->e0) != cudaSuccess ||
        cudaEventCreate(&e->e1) != cudaSuccess) {
        cudaGetLastError();
        DevFree(ctx, e->buf, e->bytes);
        if (e->h_table) cudaFreeHost(e->h_table);
        if (e->h_ids) cudaFreeHost(e->h_ids);
        if (e->h_cnt) cudaFreeHost(e->h_cnt);
        if (e->h_ctr) cudaFreeHost(e->h_ctr);
        delete e;
        return SetError(ctx, RTB200_E_OOM, "pinned host allocation failed");
    }
    std::memset(e->h_table, 0, sizeof(PtJobDev) * kMaxJobs);
    std::memset(e->h_ctr, 0, 8 * 2 * kMaxJobs);
    *out = e;
    return RTB200_OK;
}

void EngineDestroy(rtb200_engine* e)
{
    rtb200_ctx* ctx = e->ctx;
    cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < kMaxJobs; ++i)
        if (e->owner[i]) { e->owner[i]->engine = nullptr; e->owner[i]->entry = -1; }
    DropGraph(e);
    DevFree(ctx, e->buf, e->bytes);
    cudaFreeHost(e->h_table);
    cudaFreeHost(e->h_ids);
    cudaFreeHost(e->h_cnt);
    cudaFreeHost(e->h_ctr);
    cudaEventDestroy(e->e0);
    cudaEventDestroy(e->e1);
    delete e;
}

int EngineSubmit(rtb200_engine* e, rtb200_job* j, int spp)
{
    rtb200_ctx* ctx = e->ctx;
    if (spp <= 0) return SetError(ctx, RTB200_E_INVALID, "spp must be positive");
    if (j->engine) return SetError(ctx, RTB200_E_INVALID, "job is already submitted to an engine");
    if (j->scene->ctx != ctx) return SetError(ctx, RTB200_E_INVALID, "job and engine belong to different contexts");
    if (e->layout >= 0 && e->layout != j->scene->layout && !e->active.empty())
        return SetError(ctx, RTB200_E_INVALID, "all jobs of an engine must use the same BVH layout");
    int entry = -1;
    for (int i = 0; i < kMaxJobs; ++i)
        if (!e->owner[i]) { entry = i; break; }
    if (entry < 0) return SetError(ctx, RTB200_E_BUDGET, "engine job table is full");
    e->layout = j->scene->layout;
    rtb200_scene* s = j->scene;
    PtJobDev& d = e->h_table[entry];
    d.scene = PtScene{s->d_nodes, s->layout, (int)s->n_nodes, s->d_tris, (int)s->tri_material.size(), s->d_attr, s->d_mats,
                      s->d_spectra, s->d_lights, s->d_light_tris, s->d_light_nodes, s->d_light_alias,
                      s->d_tri_normals, (const PtEnvMap*)s->d_env, s->d_mesh_mat};
    d.cam = j->cam;
    d.set = j->set;
    int npx = j->npix;
    if (j->adaptive) {
        // One batch for each pixel still sampled, capped at the maximum; a
        // job with nothing left is submitted with no samples and is done at
        // once.
        spp = (int)std::max(0ll, std::min((long long)spp, (long long)j->rs.adaptive_max_spp - j->spp_done));
        npx = spp > 0 ? j->n_active : 0;
        if (npx == 0) spp = 0;
    }
    d.npix = std::max(npx, 1);
    d.px_list = j->adaptive ? j->px_list[j->cur] : nullptr;
    d.lum = j->adaptive ? j->lum : nullptr;
    d.film = j->pass;
    // Paths are counted per spectral sample: pixel sample s of a pixel is
    // paths s * spectral .. s * spectral + spectral - 1.
    d.sample_begin = (unsigned long long)j->spp_done * (unsigned long long)j->spectral;
    d.total = (unsigned long long)npx * (unsigned long long)spp * (unsigned long long)j->spectral;
    j->submitted_px = npx;
    d.sample_ctr = e->d_ctr + entry;
    d.done_ctr = e->d_ctr + kMaxJobs + entry;
    cudaMemsetAsync(e->d_ctr + entry, 0, 8, ctx->stream);
    cudaMemsetAsync(e->d_ctr + kMaxJobs + entry, 0, 8, ctx->stream);
    e->h_ctr[entry] = 0;
    e->h_ctr[kMaxJobs + entry] = 0;
    e->total[entry] = d.total;
    e->owner[entry] = j;
    e->active.push_back(entry);
    e->changed.push_back(entry);
    e->dirty = true;
    j->engine = e;
    j->entry = entry;
    j->pending_spp = spp;
    return RTB200_OK;
}

int EngineStep(rtb200_engine* e, int iterations, bool graph)
{
    rtb200_ctx* ctx = e->ctx;
    cudaStream_t st = ctx->stream;
    if (e->active.empty()) return RTB200_OK;
    if (e->fresh) {
        // Every slot starts free; statistics counters restart from zero.
        cudaMemcpyAsync(e->queues.free_, e->d_iota, 4 * (size_t)e->capacity, cudaMemcpyDeviceToDevice, st);
        int init[kCntCount] = {0};
        init[kCntFree] = e->capacity;
        std::memcpy(e->h_cnt, init, sizeof(init));
        cudaMemcpyAsync(e->queues.cnt, e->h_cnt, 4 * kCntCount, cudaMemcpyHostToDevice, st);
        e->fresh = false;
        e->seg_seen = e->shadow_seen = 0;
    }
    if (e->dirty) {
        // Upload the table entries that changed, the id list and its length.
        for (int k : e->changed)
            cudaMemcpyAsync(e->d_table + k, e->h_table + k, sizeof(PtJobDev), cudaMemcpyHostToDevice, st);
        e->changed.clear();
        for (size_t i = 0; i < e->active.size(); ++i) e->h_ids[i] = e->active[i];
        e->h_ids[kMaxJobs] = (int)e->active.size();
        cudaMemcpyAsync(e->d_ids, e->h_ids, 4 * e->active.size(), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(e->queues.cnt + kCntJobs, e->h_ids + kMaxJobs, 4, cudaMemcpyHostToDevice, st);
        e->dirty = false;
    }
    PtLaunch L = MakeLaunch(e);
    cudaError_t err = cudaSuccess;
    if (graph) {
        const rtb200_scene* us = L.uniform ? e->owner[e->active[0]]->scene : nullptr;
        if (!e->ggraph || e->glayout != L.layout || e->gspill != L.spill ||
            e->gscene != us || e->gclassify != L.classify || e->gshade_class != L.shade_class ||
            e->genv_image != L.env_image) {
            DropGraph(e);
            cudaGraph_t g = nullptr;
            err = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            PtLaunch C = L;
            for (int k = 0; k < kGraphIters && err == cudaSuccess; ++k) {
                err = PtIteration(C, k, st);
                std::swap(C.queues.active, C.queues.active_next);
                std::swap(C.queues.free_, C.queues.free_next);
            }
            const cudaError_t e2 = cudaStreamEndCapture(st, &g);
            if (err == cudaSuccess) err = e2;
            if (err == cudaSuccess) err = cudaGraphInstantiate(&e->gexec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (err != cudaSuccess) { DropGraph(e); return CudaCheck(ctx, err, "graph capture"); }
            e->ggraph = true;
            e->glayout = L.layout;
            e->gspill = L.spill;
            e->gscene = us;
            e->gclassify = L.classify;
            e->genv_image = L.env_image;
            e->gshade_class = L.shade_class;
        }
        const int reps = (iterations + kGraphIters - 1) / kGraphIters;
        for (int r = 0; r < reps && err == cudaSuccess; ++r) err = cudaGraphLaunch(e->gexec, st);
        e->iter += reps * kGraphIters;
    } else {
        // Direct launches; an even count keeps the queue buffers where the
        // captured graph expects them.
        const int n = ((iterations + 1) / 2) * 2;
        for (int k = 0; k < n && err == cudaSuccess; ++k) {
            err = PtIteration(L, e->iter++, st);
            std::swap(L.queues.active, L.queues.active_next);
            std::swap(L.queues.free_, L.queues.free_next);
        }
    }
    for (size_t a = 0; a < e->active.size() && err == cudaSuccess; ++a) {
        rtb200_job* j = e->owner[e->active[a]];
        if (j->pending_spp < kFoldEverySpp) continue;
        err = j->wide ? PtFoldWide(j->pass, j->sum, j->comp, j->wide, j->film_n, false, ctx->num_sms, st)
                      : PtFold(j->pass, j->sum, j->comp, j->film_n, ctx->num_sms, st);
    }
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(e->h_cnt, e->queues.cnt, 4 * kCntCount, cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaMemcpyAsync(e->h_ctr, e->d_ctr, 8 * 2 * kMaxJobs, cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) return CudaCheck(ctx, err, "wavefront step");
    unsigned errw = 0;
    cudaMemcpy(&errw, e->queues.err, 4, cudaMemcpyDeviceToHost);
    if (errw) return SetError(ctx, RTB200_E_DEVICE, "device error word set (traversal stack overflow)");
    // Per-job statistics: attribute this step's segments to the active jobs.
    const long long seg = (unsigned)e->h_cnt[kCntSegments], sh = (unsigned)e->h_cnt[kCntShadowRays];
    const long long dseg = seg - e->seg_seen, dsh = sh - e->shadow_seen;
    e->seg_seen = seg;
    e->shadow_seen = sh;
    if (!e->active.empty()) {
        for (int id : e->active) {
            e->owner[id]->segments += dseg / (long long)e->active.size();
            e->owner[id]->shadow_rays += dsh / (long long)e->active.size();
        }
    }
    return RTB200_OK;
}

bool JobDone(const rtb200_engine* e, int entry) { return e->h_ctr[kMaxJobs + entry] >= e->total[entry]; }

// Cuts a job's request in flight to the pixel samples already started: its
// total becomes the paths issued so far (exact: the device is idle after a
// step) rounded up to whole pixel samples, so every pixel ends with the same
// count; the table change reaches the device before the next step's
// KAssign.
void CancelEntry(rtb200_engine* e, rtb200_job* j)
{
    const int entry = j->entry;
    const unsigned long long unit = (unsigned long long)std::max(j->submitted_px, 1) * (unsigned long long)j->spectral;
    unsigned long long t = (e->h_ctr[entry] + unit - 1) / unit * unit;
    if (t > e->total[entry]) t = e->total[entry];
    e->total[entry] = t;
    e->h_table[entry].total = t;
    e->changed.push_back(entry);
    e->dirty = true;
    j->pending_spp = (long long)(t / unit);
}

int EngineRetire(rtb200_engine* e, rtb200_job* j)
{
    rtb200_ctx* ctx = e->ctx;
    if (j->engine != e) return SetError(ctx, RTB200_E_INVALID, "job is not submitted to this engine");
    if (!JobDone(e, j->entry)) return SetError(ctx, RTB200_E_NOT_READY, "job still has samples in flight");
    // Past kWideSpp samples per pixel the running sum moves to FP64.
    cudaError_t err;
    if (!j->wide && j->spp_done + j->pending_spp > kWideSpp) {
        void* w = nullptr;
        const int rc = DevAllocCached(ctx, &w, 8 * (size_t)j->film_n);
        if (rc) return rc;
        j->wide = (double*)w;
        err = PtFoldWide(j->pass, j->sum, j->comp, j->wide, j->film_n, true, ctx->num_sms, ctx->stream);
    } else if (j->wide) {
        err = PtFoldWide(j->pass, j->sum, j->comp, j->wide, j->film_n, false, ctx->num_sms, ctx->stream);
    } else {
        err = PtFold(j->pass, j->sum, j->comp, j->film_n, ctx->num_sms, ctx->stream);
    }
    if (err != cudaSuccess) return CudaCheck(ctx, err, "film fold");
    if (j->adaptive && j->pending_spp > 0 && j->submitted_px > 0) {
        err = PtConverge(j->px_list[j->cur], j->submitted_px, j->lum, j->counts, (int)j->pending_spp,
                         j->rs.adaptive_max_spp, (double)j->rs.adaptive_threshold, j->px_list[j->cur ^ 1], j->d_n,
                         ctx->num_sms, ctx->stream);
        int n = 0;
        if (err == cudaSuccess) err = cudaMemcpyAsync(&n, j->d_n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
        if (err != cudaSuccess) return CudaCheck(ctx, err, "adaptive convergence");
        j->cur ^= 1;
        j->n_active = n;
    }
    j->spp_done += j->pending_spp;
    j->samples += (long long)j->submitted_px * j->pending_spp;
    j->pending_spp = 0;
    const int entry = j->entry;
    e->active.erase(std::find(e->active.begin(), e->active.end(), entry));
    e->owner[entry] = nullptr;
    e->total[entry] = 0;
    e->h_table[entry].total = 0;
    e->changed.push_back(entry);
    e->dirty = true;
    j->engine = nullptr;
    j->entry = -1;
    return RTB200_OK;
}

// Submit all, step until every job is done, retire all.
int EngineRender(rtb200_engine* e, rtb200_job* const* jobs, const int32_t* spp, int n, bool graph)
{
    rtb200_ctx* ctx = e->ctx;
    for (int i = 0; i < n; ++i) {
        const int rc = EngineSubmit(e, jobs[i], spp[i]);
        if (rc) {
            for (int k = 0; k < i; ++k) {
                // Undo earlier submissions: nothing has run yet.
                rtb200_job* j = jobs[k];
                e->active.erase(std::find(e->active.begin(), e->active.end(), j->entry));
                e->owner[j->entry] = nullptr;
                e->total[j->entry] = 0;
                j->engine = nullptr;
                j->entry = -1;
            }
            e->dirty = true;
            return rc;
        }
    }
    cudaEventRecord(e->e0, ctx->stream);
    const long long kMaxSteps = 1ll << 18;
    std::vector<char> cancelled((size_t)n, 0);
    bool any_cancel = false;
    for (long long step = 0;; ++step) {
        const int rc = EngineStep(e, e->poll, graph);
        if (rc) return rc;
        for (int i = 0; i < n; ++i) {
            rtb200_job* j = jobs[i];
            if (!j->progress || cancelled[i]) continue;
            const double unit = (double)std::max(j->submitted_px, 1) * (double)j->spectral;
            const double done = (double)e->h_ctr[kMaxJobs + j->entry] / unit, tot = (double)e->total[j->entry] / unit;
            if (!j->progress(j->progress_user, done, tot)) {
                CancelEntry(e, j);
                cancelled[i] = 1;
                any_cancel = true;
            }
        }
        bool all = true;
        for (int i = 0; i < n; ++i) all = all && JobDone(e, jobs[i]->entry);
        if (all) break;
        if (step > kMaxSteps) return SetError(ctx, RTB200_E_TIMEOUT, "render did not finish its samples");
    }
    cudaEventRecord(e->e1, ctx->stream);
    cudaEventSynchronize(e->e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e->e0, e->e1);
    for (int i = 0; i < n; ++i) {
        jobs[i]->seconds += ms * 1e-3;
        const int rc = EngineRetire(e, jobs[i]);
        if (rc) return rc;
    }
    const int rc = CudaCheck(ctx, cudaStreamSynchronize(ctx->stream), "film fold");
    if (rc) return rc;
    return any_cancel ? SetError(ctx, RTB200_E_CANCELLED, "stopped by the progress callback") : RTB200_OK;
}

}  // namespace

extern "C" {

int rtb200_job_create(rtb200_scene* s, const rtb200_render_settings* rs, rtb200_job** out)
{
    if (!s || !rs || !out) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    *out = nullptr;
    if (!s->committed || s->materials.empty())
        return SetError(ctx, RTB200_E_INVALID, "scene must be committed with materials");
    if (s->layout == RTB200_BVH_W8)
        return SetError(ctx, RTB200_E_INVALID, "the path tracer runs on the four-wide BVH layouts (F32, Q8, F16)");
    if (rs->width <= 0 || rs->height <= 0 || (int64_t)rs->width * rs->height > (1ll << 28) || rs->max_depth < 1 ||
        rs->max_depth > 255 || !(rs->lambda_max > rs->lambda_min) || rs->lambda_min < 380.0f ||
        rs->lambda_max > 780.0f || !(rs->fov_deg > 0.0f && rs->fov_deg < 180.0f))
        return SetError(ctx, RTB200_E_INVALID, "bad render settings");
    if (rs->filter != RTB200_FILTER_BOX &&
        !(rs->filter == RTB200_FILTER_GAUSSIAN && rs->filter_size > 0.0f && rs->filter_size <= 16.0f &&
          rs->filter_sigma > 0.0f))
        return SetError(ctx, RTB200_E_INVALID, "bad pixel filter settings");
    if (rs->light_selection != RTB200_LIGHTS_BVH && rs->light_selection != RTB200_LIGHTS_POWER)
        return SetError(ctx, RTB200_E_INVALID, "bad light selection");
    if (rs->adaptive_max_spp < 0 || (rs->adaptive_max_spp > 0 && !(rs->adaptive_threshold > 0.0f)))
        return SetError(ctx, RTB200_E_INVALID, "bad adaptive sampling settings");
    if (rs->sampler != RTB200_SAMPLER_HASH && rs->sampler != RTB200_SAMPLER_SOBOL &&
        rs->sampler != RTB200_SAMPLER_SOBOL_SHUFFLED)
        return SetError(ctx, RTB200_E_INVALID, "bad sampler");
    if (rs->bounce_limits && (rs->max_diffuse_bounce < 0 || rs->max_glossy_bounce < 0 ||
                              rs->max_transmission_bounce < 0))
        return SetError(ctx, RTB200_E_INVALID, "bad bounce limits");
    if ((rs->spectral_mode != RTB200_SPECTRAL_HWSS && rs->spectral_mode != RTB200_SPECTRAL_SINGLE) ||
        rs->num_wavelengths < 0 || rs->spectral_samples < 0 || rs->spectral_samples > 256)
        return SetError(ctx, RTB200_E_INVALID, "bad spectral settings");
    if (rs->spectral_samples > 1 && rs->adaptive_max_spp > 0)
        return SetError(ctx, RTB200_E_INVALID, "adaptive sampling needs one spectral sample per pixel sample");
    // Camera frame (pinhole; vertical field of view).
    const float* P = rs->cam_pos;
    double f[3] = {rs->cam_look[0] - P[0], rs->cam_look[1] - P[1], rs->cam_look[2] - P[2]};
    const double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    if (!(fl > 0.0)) return SetError(ctx, RTB200_E_INVALID, "degenerate camera frame");
    for (double& x : f) x /= fl;
    const double u[3] = {rs->cam_up[0], rs->cam_up[1], rs->cam_up[2]};
    double r[3] = {f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0]};
    const double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (!(rl > 0.0)) return SetError(ctx, RTB200_E_INVALID, "degenerate camera frame");
    for (double& x : r) x /= rl;
    const double uu[3] = {r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]};
    cudaSetDevice(ctx->device);
    rtb200_job* j = new (std::nothrow) rtb200_job();
    if (!j) return SetError(ctx, RTB200_E_OOM, "host allocation failed");
    j->scene = s;
    j->rs = *rs;
    j->npix = rs->width * rs->height;
    const double th = std::tan(0.5 * rs->fov_deg * 3.14159265358979323846 / 180.0);
    const double aspect = (double)rs->width / (double)rs->height;
    for (int k = 0; k < 3; ++k) {
        j->cam.pos[k] = P[k];
        j->cam.fwd[k] = (float)f[k];
        j->cam.right[k] = (float)(r[k] * th * aspect);
        j->cam.up[k] = (float)(uu[k] * th);
    }
    j->cam.width = rs->width;
    j->cam.height = rs->height;
    PtSettings& st = j->set;
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
    st.light_bvh = rs->light_selection == RTB200_LIGHTS_BVH ? 1 : 0;
    st.sampler = rs->sampler == RTB200_SAMPLER_SOBOL ? kSamplerSobol
                 : rs->sampler == RTB200_SAMPLER_SOBOL_SHUFFLED ? kSamplerSobolShuffled : kSamplerHash;
    {
        // Counts are kept in a byte each and a path has at most 255 vertices,
        // so 255 means no limit.
        const int32_t lim[3] = {rs->max_diffuse_bounce, rs->max_glossy_bounce, rs->max_transmission_bounce};
        for (int k = 0; k < 3; ++k) st.max_bounce[k] = rs->bounce_limits ? std::min(lim[k], 255) : 255;
    }
    st.single = rs->spectral_mode == RTB200_SPECTRAL_SINGLE ? 1 : 0;
    st.num_wl = rs->num_wavelengths > 0 && rs->num_wavelengths < 10000 ? rs->num_wavelengths : 0;
    st.wl_step = st.num_wl ? (float)(((double)rs->lambda_max - rs->lambda_min) / st.num_wl) : 0.0f;
    j->spectral = std::max(1, (int)rs->spectral_samples);
    st.inv_spectral = 1.0f / (float)j->spectral;
    const bool gauss = rs->filter == RTB200_FILTER_GAUSSIAN;
    st.filter = !gauss ? kFilterBox : (0.5 * rs->filter_size > 0.501 ? kFilterSplat : kFilterWarp);
    st.filt_half = gauss ? 0.5f * rs->filter_size : 0.5f;
    st.filt_inv2s2 = gauss ? 1.0f / (2.0f * rs->filter_sigma * rs->filter_sigma) : 0.0f;
    st.filt_norm = gauss ? (float)(1.0 / (3.14159265358979323846 * 2.0 * rs->filter_sigma * rs->filter_sigma)) : 1.0f;
    st.filt_sigma = gauss ? rs->filter_sigma : 0.0f;
    {
        const double k = gauss ? 0.5 * rs->filter_size / rs->filter_sigma : 0.0;
        st.filt_trunc = (float)std::exp(-0.5 * k * k);
    }
    // Film: this request's accumulator, running sum, Kahan compensation; XYZ
    // per pixel, plus the weight sum for splatted films.
    j->channels = st.filter == kFilterSplat ? 4 : 3;
    j->film_n = j->channels * j->npix;
    const size_t plane = Align(4 * (size_t)j->film_n);
    int rc = DevAllocCached(ctx, &j->film_buf, 3 * plane);
    if (rc) { delete j; return rc; }
    j->film_bytes = 3 * plane;
    // Stream-ordered: a reused block may still be read by earlier work.
    cudaMemsetAsync(j->film_buf, 0, 3 * plane, ctx->stream);
    j->pass = (float*)j->film_buf;
    j->sum = (float*)((char*)j->film_buf + plane);
    j->comp = (float*)((char*)j->film_buf + 2 * plane);
    j->n_active = j->npix;
    if (rs->adaptive_max_spp > 0) {
        // Pixel lists (two), sample counts, luminance sums, list length.
        const size_t pl = Align(4 * (size_t)j->npix), pc = Align(4 * (size_t)j->npix),
                     ps = Align(16 * (size_t)j->npix);
        j->adapt_bytes = 2 * pl + pc + ps + 256;
        rc = DevAllocCached(ctx, &j->adapt_buf, j->adapt_bytes);
        if (rc) {
            DevFreeCached(ctx, j->film_buf, j->film_bytes);
            delete j;
            return rc;
        }
        char* b = (char*)j->adapt_buf;
        j->px_list[0] = (unsigned*)b;
        j->px_list[1] = (unsigned*)(b + pl);
        j->counts = (unsigned*)(b + 2 * pl);
        j->lum = (double*)(b + 2 * pl + pc);
        j->d_n = (int*)(b + 2 * pl + pc + ps);
        j->adaptive = true;
        std::vector<unsigned> all((size_t)j->npix);
        for (size_t i = 0; i < all.size(); ++i) all[i] = (unsigned)i;
        cudaError_t err = cudaMemsetAsync(j->counts, 0, pc + ps, ctx->stream);
        // From pageable memory: returns once the host buffer has been staged.
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(j->px_list[0], all.data(), 4 * all.size(), cudaMemcpyHostToDevice, ctx->stream);
        if (err != cudaSuccess) {
            DevFreeCached(ctx, j->adapt_buf, j->adapt_bytes);
            DevFreeCached(ctx, j->film_buf, j->film_bytes);
            delete j;
            return CudaCheck(ctx, err, "adaptive sampling set-up");
        }
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
    if (j->engine) return SetError(ctx, RTB200_E_INVALID, "job is submitted to an engine");
    cudaSetDevice(ctx->device);
    if (!j->own) {
        int cap = j->rs.max_paths > 0 ? j->rs.max_paths : std::min(std::max(j->npix * 8, 65536), 1 << 21);
        const int rc = EngineCreate(ctx, cap, &j->own);
        if (rc) return rc;
    }
    rtb200_job* list[1] = {j};
    const int32_t s[1] = {spp};
    return EngineRender(j->own, list, s, 1, false);
}

int rtb200_job_read_film(rtb200_job* j, float* xyz)
{
    if (!j || !xyz) return RTB200_E_INVALID;
    rtb200_ctx* ctx = j->scene->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (j->engine) return SetError(ctx, RTB200_E_NOT_READY, "job has a request in flight");
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)j->film_n;
    std::vector<double> acc(n);
    if (j->wide) {
        const cudaError_t e = cudaMemcpy(acc.data(), j->wide, 8 * n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return CudaCheck(ctx, e, "film readback");
    } else {
        std::vector<float> sum(n), comp(n);
        cudaError_t e = cudaMemcpy(sum.data(), j->sum, 4 * n, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(comp.data(), j->comp, 4 * n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return CudaCheck(ctx, e, "film readback");
        for (size_t i = 0; i < n; ++i) acc[i] = (double)sum[i] - (double)comp[i];
    }
    if (j->channels == 3 && j->adaptive) {
        std::vector<unsigned> cnt((size_t)j->npix);
        const cudaError_t e = cudaMemcpy(cnt.data(), j->counts, 4 * cnt.size(), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return CudaCheck(ctx, e, "film readback");
        for (size_t i = 0; i < n; ++i) xyz[i] = cnt[i / 3] ? (float)(acc[i] / (double)cnt[i / 3]) : 0.0f;
    } else if (j->channels == 3) {
        const double inv = j->spp_done > 0 ? 1.0 / (double)j->spp_done : 0.0;
        for (size_t i = 0; i < n; ++i) xyz[i] = (float)(acc[i] * inv);
    } else {
        // FilteredFilm resolve (Rendering/FilteredFilm.cpp:100-132): weighted
        // sum over the weight; pixels no sample reached stay 0.
        for (size_t p = 0; p < (size_t)j->npix; ++p) {
            const double w = acc[4 * p + 3];
            for (int c = 0; c < 3; ++c) xyz[3 * p + c] = std::fabs(w) > 1e-10 ? (float)(acc[4 * p + c] / w) : 0.0f;
        }
    }
    return RTB200_OK;
}

int rtb200_job_relmse(rtb200_job* j, const float* ref_xyz, double* relmse)
{
    if (!j || !ref_xyz || !relmse) return RTB200_E_INVALID;
    rtb200_ctx* ctx = j->scene->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (j->engine) return SetError(ctx, RTB200_E_NOT_READY, "job has a request in flight");
    cudaSetDevice(ctx->device);
    const size_t n3 = 3 * (size_t)j->npix;
    void* buf = nullptr;
    int rc = DevAllocCached(ctx, &buf, Align(4 * n3) + 8);
    if (rc) return rc;
    float* d_ref = (float*)buf;
    double* d_out = (double*)((char*)buf + Align(4 * n3));
    double sum = 0.0;
    cudaError_t e = cudaMemcpyAsync(d_ref, ref_xyz, 4 * n3, cudaMemcpyHostToDevice, ctx->stream);
    const double inv = j->spp_done > 0 ? 1.0 / (double)j->spp_done : 0.0;
    if (e == cudaSuccess)
        e = PtRelMse(j->sum, j->comp, j->wide, j->adaptive ? j->counts : nullptr, d_ref, j->npix, j->channels, inv,
                     d_out, ctx->num_sms, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&sum, d_out, 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    DevFreeCached(ctx, buf, Align(4 * n3) + 8);
    if (e != cudaSuccess) return CudaCheck(ctx, e, "relMSE");
    *relmse = sum / (double)n3;
    return RTB200_OK;
}

int rtb200_job_read_sample_counts(rtb200_job* j, uint32_t* counts)
{
    if (!j || !counts) return RTB200_E_INVALID;
    rtb200_ctx* ctx = j->scene->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (j->engine) return SetError(ctx, RTB200_E_NOT_READY, "job has a request in flight");
    if (!j->adaptive) {
        std::fill(counts, counts + j->npix, (uint32_t)j->spp_done);
        return RTB200_OK;
    }
    cudaSetDevice(ctx->device);
    return CudaCheck(ctx, cudaMemcpy(counts, j->counts, 4 * (size_t)j->npix, cudaMemcpyDeviceToHost),
                     "sample count readback");
}

namespace {
// Resolve the film on the device into a temporary buffer and copy it out.
int ReadColor(rtb200_job* j, double ev_mul, int tone, float* rgb, uint8_t* rgb8)
{
    rtb200_ctx* ctx = j->scene->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (j->engine) return SetError(ctx, RTB200_E_NOT_READY, "job has a request in flight");
    cudaSetDevice(ctx->device);
    const size_t bytes = (rgb ? 12 : 3) * (size_t)j->npix;
    void* buf = nullptr;
    const int rc = DevAllocCached(ctx, &buf, Align(bytes));
    if (rc) return rc;
    const double inv = j->spp_done > 0 ? 1.0 / (double)j->spp_done : 0.0;
    cudaError_t e = PtResolveColor(j->sum, j->comp, j->wide, j->adaptive ? j->counts : nullptr, j->channels, inv,
                                   j->npix, ev_mul, tone, rgb ? (float*)buf : nullptr,
                                   rgb ? nullptr : (unsigned char*)buf, ctx->num_sms, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(rgb ? (void*)rgb : (void*)rgb8, buf, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    DevFreeCached(ctx, buf, Align(bytes));
    return CudaCheck(ctx, e, "colour resolve");
}
}  // namespace

int rtb200_job_read_rgb(rtb200_job* j, float* rgb)
{
    if (!j || !rgb) return RTB200_E_INVALID;
    return ReadColor(j, 1.0, RTB200_TONE_NONE, rgb, nullptr);
}

int rtb200_job_read_display(rtb200_job* j, float exposure_ev, int32_t tone, uint8_t* rgb8)
{
    if (!j || !rgb8) return RTB200_E_INVALID;
    if (tone < RTB200_TONE_NONE || tone > RTB200_TONE_HABLE || !std::isfinite(exposure_ev))
        return SetError(j->scene->ctx, RTB200_E_INVALID, "bad display settings");
    return ReadColor(j, std::pow(2.0, (double)exposure_ev), tone, nullptr, rgb8);
}

int rtb200_job_stats(const rtb200_job* j, rtb200_stats* out)
{
    if (!j || !out) return RTB200_E_INVALID;
    out->active_pixels = j->adaptive ? (j->spp_done < j->rs.adaptive_max_spp ? j->n_active : 0) : j->npix;
    out->spp = j->spp_done;
    out->samples = j->samples;
    out->segments = j->segments;
    out->shadow_rays = j->shadow_rays;
    out->seconds = j->seconds;
    return RTB200_OK;
}

int rtb200_job_destroy(rtb200_job* j)
{
    if (!j) return RTB200_E_INVALID;
    rtb200_ctx* ctx = j->scene->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (j->engine) return SetError(ctx, RTB200_E_NOT_READY, "retire the job from its engine first");
    cudaSetDevice(ctx->device);
    if (j->own) EngineDestroy(j->own);   // synchronises the stream
    // The film goes back to the context's cache; work still queued on the
    // stream finishes before any later user of the block runs.
    DevFreeCached(ctx, j->film_buf, j->film_bytes);
    if (j->wide) DevFreeCached(ctx, j->wide, 8 * (size_t)j->film_n);
    if (j->adapt_buf) DevFreeCached(ctx, j->adapt_buf, j->adapt_bytes);
    delete j;
    return RTB200_OK;
}

int rtb200_engine_create(rtb200_ctx* ctx, int32_t capacity, rtb200_engine** out)
{
    if (!ctx || !out || capacity < 0) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return EngineCreate(ctx, capacity, out);
}

int rtb200_engine_render(rtb200_engine* e, rtb200_job* const* jobs, const int32_t* spp, int32_t n, int32_t use_graph)
{
    if (!e || n < 0 || (n > 0 && (!jobs || !spp))) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(e->ctx->mu);
    for (int i = 0; i < n; ++i)
        if (!jobs[i]) return SetError(e->ctx, RTB200_E_INVALID, "null job");
    cudaSetDevice(e->ctx->device);
    return EngineRender(e, jobs, spp, n, use_graph != 0);
}

int rtb200_engine_submit(rtb200_engine* e, rtb200_job* job, int32_t spp)
{
    if (!e || !job) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(e->ctx->mu);
    cudaSetDevice(e->ctx->device);
    return EngineSubmit(e, job, spp);
}

int rtb200_engine_step(rtb200_engine* e, int32_t iterations, int32_t use_graph)
{
    if (!e || iterations <= 0) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(e->ctx->mu);
    cudaSetDevice(e->ctx->device);
    return EngineStep(e, iterations, use_graph != 0);
}

int rtb200_engine_progress(const rtb200_engine* e, const rtb200_job* job, int64_t* done, int64_t* total)
{
    if (!e || !job || job->engine != e) return RTB200_E_INVALID;
    if (done) *done = (int64_t)e->h_ctr[kMaxJobs + job->entry];
    if (total) *total = (int64_t)e->total[job->entry];
    return RTB200_OK;
}

int rtb200_engine_retire(rtb200_engine* e, rtb200_job* job)
{
    if (!e || !job) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(e->ctx->mu);
    cudaSetDevice(e->ctx->device);
    const int rc = EngineRetire(e, job);
    if (rc) return rc;
    return CudaCheck(e->ctx, cudaStreamSynchronize(e->ctx->stream), "film fold");
}

int rtb200_engine_cancel(rtb200_engine* e, rtb200_job* job)
{
    if (!e || !job) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(e->ctx->mu);
    if (job->engine != e) return SetError(e->ctx, RTB200_E_INVALID, "job is not submitted to this engine");
    CancelEntry(e, job);
    return RTB200_OK;
}

int rtb200_job_set_progress(rtb200_job* job, rtb200_progress_fn fn, void* user)
{
    if (!job) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(job->scene->ctx->mu);
    job->progress = fn;
    job->progress_user = user;
    return RTB200_OK;
}

int rtb200_engine_set_poll(rtb200_engine* e, int32_t iterations)
{
    if (!e) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(e->ctx->mu);
    if (iterations < 1 || iterations > 1024) return SetError(e->ctx, RTB200_E_INVALID, "poll interval out of range");
    e->poll = (iterations + 1) & ~1;
    return RTB200_OK;
}

int rtb200_engine_destroy(rtb200_engine* e)
{
    if (!e) return RTB200_E_INVALID;
    rtb200_ctx* ctx = e->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    EngineDestroy(e);
    return RTB200_OK;
}

}  // extern "C"
