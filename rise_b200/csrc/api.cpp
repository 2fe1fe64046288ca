// api.cpp -- the C ABI (include/rtb200.h): contexts, scenes, batched casts.
//
// Ownership follows the reference's explicit create/release style
// (src/Library/Interfaces/IReference.h) with opaque handles; failures return
// a status code and leave a message in rtb200_last_error instead of logging.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>

#include "core.h"

namespace rtb200 {

int SetError(rtb200_ctx* ctx, int code, const std::string& msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

int CudaCheck(rtb200_ctx* ctx, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return RTB200_OK;
    return SetError(ctx, e == cudaErrorMemoryAllocation ? RTB200_E_OOM : RTB200_E_DEVICE,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

int DevAlloc(rtb200_ctx* ctx, void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) return RTB200_OK;
    if (ctx->budget && ctx->in_use + ctx->cached + bytes > ctx->budget) DevReleaseCache(ctx);
    if (ctx->budget && ctx->in_use + bytes > ctx->budget)
        return SetError(ctx, RTB200_E_BUDGET, "device memory budget exceeded");
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation && ctx->cached) {
        cudaGetLastError();
        DevReleaseCache(ctx);
        e = cudaMalloc(p, bytes);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return SetError(ctx, RTB200_E_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    ctx->in_use += bytes;
    return RTB200_OK;
}

void DevFree(rtb200_ctx* ctx, void* p, size_t bytes)
{
    if (!p) return;
    cudaFree(p);
    ctx->in_use -= bytes;
}

int DevAllocCached(rtb200_ctx* ctx, void** p, size_t bytes)
{
    auto it = ctx->cache.find(bytes);
    if (it != ctx->cache.end() && !it->second.empty()) {
        if (ctx->budget && ctx->in_use + bytes > ctx->budget)
            return SetError(ctx, RTB200_E_BUDGET, "device memory budget exceeded");
        *p = it->second.back();
        it->second.pop_back();
        ctx->cached -= bytes;
        ctx->in_use += bytes;
        return RTB200_OK;
    }
    return DevAlloc(ctx, p, bytes);
}

void DevFreeCached(rtb200_ctx* ctx, void* p, size_t bytes)
{
    if (!p) return;
    if (ctx->cached + bytes > kDevCacheBytes) {
        DevFree(ctx, p, bytes);
        return;
    }
    ctx->cache[bytes].push_back(p);
    ctx->cached += bytes;
    ctx->in_use -= bytes;
}

void DevReleaseCache(rtb200_ctx* ctx)
{
    if (!ctx->cached) return;
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->cache)
        for (void* q : kv.second) cudaFree(q);
    ctx->cache.clear();
    ctx->cached = 0;
}

namespace {

int EnsureStage(rtb200_scene* s, size_t in_bytes, size_t out_bytes)
{
    rtb200_ctx* ctx = s->ctx;
    if (in_bytes > s->stage_in) {
        DevFree(ctx, s->d_in, s->stage_in);
        s->d_in = nullptr;
        s->stage_in = 0;
        int rc = DevAlloc(ctx, &s->d_in, in_bytes);
        if (rc) return rc;
        s->stage_in = in_bytes;
    }
    if (out_bytes > s->stage_out) {
        DevFree(ctx, s->d_out, s->stage_out);
        s->d_out = nullptr;
        s->stage_out = 0;
        int rc = DevAlloc(ctx, &s->d_out, out_bytes);
        if (rc) return rc;
        s->stage_out = out_bytes;
    }
    return RTB200_OK;
}

// Host-buffer casts in chunks: the upload of chunk k+1 (copy_in stream) and
// the download of chunk k-1 (copy_out stream) overlap the trace of chunk k,
// with two staging buffers each way and events ordering their reuse.  Chunks
// alternate between two trace streams (ctx->stream, ctx->trace2), each launch
// with its own work counter, so one chunk's blocks start while the previous
// chunk's last rays finish instead of the device idling in every launch's tail.
// `trace(d_in, m, d_out, counter, stream)` launches the kernel on m staged rays.
template <class Trace>
cudaError_t PipelinedCast(rtb200_scene* s, const rtb200_ray* rays, int64_t n, void* out, size_t out_bytes_per_ray,
                          int& rc, Trace trace)
{
    rtb200_ctx* ctx = s->ctx;
    const int64_t chunk = std::max<int64_t>(std::min<int64_t>(n, int64_t(1) << 18), (n + 7) / 8);
    const int nbuf = n > chunk ? 2 : 1;
    rc = EnsureStage(s, (size_t)nbuf * chunk * sizeof(rtb200_ray), (size_t)nbuf * chunk * out_bytes_per_ray);
    if (rc) return cudaSuccess;
    cudaStream_t ts[2] = {ctx->stream, ctx->trace2};
    // Work counters of the two trace streams (scene scratch bytes 128 and 192).
    unsigned long long* counter[2] = {(unsigned long long*)((char*)s->d_counter + 128),
                                      (unsigned long long*)((char*)s->d_counter + 192)};
    // Everything after the work already queued on ctx->stream.
    cudaError_t e = cudaEventRecord(ctx->ev_trace[0], ts[0]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_in, ctx->ev_trace[0], 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ts[1], ctx->ev_trace[0], 0);
    const int64_t nchunks = (n + chunk - 1) / chunk;
    for (int64_t k = 0; k < nchunks && e == cudaSuccess; ++k) {
        const int b = (int)(k & 1);
        const int64_t off = k * chunk, m = std::min(chunk, n - off);
        rtb200_ray* d_in = (rtb200_ray*)s->d_in + b * chunk;
        char* d_out = (char*)s->d_out + (size_t)b * chunk * out_bytes_per_ray;
        if (k >= 2) e = cudaStreamWaitEvent(ctx->copy_in, ctx->ev_trace[b], 0);   // chunk k-2 traced
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_in, rays + off, (size_t)m * sizeof(rtb200_ray), cudaMemcpyHostToDevice, ctx->copy_in);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_up[b], ctx->copy_in);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ts[b], ctx->ev_up[b], 0);
        if (e == cudaSuccess && k >= 2) e = cudaStreamWaitEvent(ts[b], ctx->ev_down[b], 0);   // chunk k-2 downloaded
        if (e == cudaSuccess) e = cudaMemsetAsync(counter[b], 0, sizeof(unsigned long long), ts[b]);
        if (e == cudaSuccess) e = trace(d_in, m, d_out, counter[b], ts[b]);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_trace[b], ts[b]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_out, ctx->ev_trace[b], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync((char*)out + (size_t)off * out_bytes_per_ray, d_out, (size_t)m * out_bytes_per_ray,
                                cudaMemcpyDeviceToHost, ctx->copy_out);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_down[b], ctx->copy_out);
    }
    // Later work on ctx->stream waits for both trace streams and the downloads.
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_trace[1], ts[1]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ts[0], ctx->ev_trace[1], 0);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_down[0], ctx->copy_out);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ts[0], ctx->ev_down[0], 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ts[0]);
    return e;
}

int CheckErrWord(rtb200_scene* s, cudaStream_t st)
{
    unsigned err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, s->d_err, sizeof(err), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return CudaCheck(s->ctx, e, "error word readback");
    if (err) {
        cudaMemsetAsync(s->d_err, 0, sizeof(unsigned), st);
        return SetError(s->ctx, RTB200_E_DEVICE, "device error word set (traversal stack overflow)");
    }
    return RTB200_OK;
}

bool Aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace
}  // namespace rtb200

using namespace rtb200;

extern "C" {

int rtb200_ctx_create(int device, size_t budget_bytes, rtb200_ctx** out)
{
    if (!out) return RTB200_E_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return RTB200_E_DEVICE;
    }
    rtb200_ctx* ctx = new (std::nothrow) rtb200_ctx();
    if (!ctx) return RTB200_E_OOM;
    ctx->device = device;
    ctx->budget = budget_bytes;
    bool ok = cudaSetDevice(device) == cudaSuccess &&
              cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
              cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&ctx->trace2, cudaStreamNonBlocking) == cudaSuccess;
    for (int b = 0; b < 2 && ok; ++b)
        ok = cudaEventCreateWithFlags(&ctx->ev_up[b], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&ctx->ev_trace[b], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&ctx->ev_down[b], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        delete ctx;
        return RTB200_E_DEVICE;
    }
    *out = ctx;
    return RTB200_OK;
}

int rtb200_ctx_destroy(rtb200_ctx* ctx)
{
    if (!ctx) return RTB200_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    DevReleaseCache(ctx);
    for (int b = 0; b < 2; ++b) {
        cudaEventDestroy(ctx->ev_up[b]);
        cudaEventDestroy(ctx->ev_trace[b]);
        cudaEventDestroy(ctx->ev_down[b]);
    }
    cudaStreamDestroy(ctx->copy_in);
    cudaStreamDestroy(ctx->copy_out);
    cudaStreamDestroy(ctx->trace2);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return RTB200_OK;
}

const char* rtb200_last_error(const rtb200_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

size_t rtb200_ctx_bytes_in_use(const rtb200_ctx* ctx) { return ctx ? ctx->in_use : 0; }

int rtb200_scene_create(rtb200_ctx* ctx, rtb200_scene** out)
{
    if (!ctx || !out) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    *out = nullptr;
    rtb200_scene* s = new (std::nothrow) rtb200_scene();
    if (!s) return SetError(ctx, RTB200_E_OOM, "host allocation failed");
    s->ctx = ctx;
    cudaSetDevice(ctx->device);
    void* p = nullptr;
    int rc = DevAlloc(ctx, &p, 256);
    if (rc) { delete s; return rc; }
    cudaMemset(p, 0, 256);
    s->d_counter = (unsigned long long*)p;
    s->d_err = (unsigned*)((char*)p + 64);
    *out = s;
    return RTB200_OK;
}

static int AddMesh(rtb200_scene* s, const float* xyz, int64_t n_verts, const uint32_t* tri, int64_t n_tri,
            const float* nrm, int64_t n_nrm, const uint32_t* tri_nrm, int32_t material, int32_t double_sided)
{
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (s->committed) return SetError(ctx, RTB200_E_INVALID, "scene already committed");
    if (n_verts < 0 || n_tri < 0 || (n_tri > 0 && (!xyz || !tri)))
        return SetError(ctx, RTB200_E_INVALID, "bad mesh arguments");
    if (nrm && (n_nrm < 0 || (n_tri > 0 && !tri_nrm)))
        return SetError(ctx, RTB200_E_INVALID, "bad normal arguments");
    if ((int64_t)(s->tri_material.size()) + n_tri > (int64_t)INT32_MAX)
        return SetError(ctx, RTB200_E_INVALID, "too many triangles");
    for (int64_t i = 0; i < 3 * n_tri; ++i)
        if ((int64_t)tri[i] >= n_verts) return SetError(ctx, RTB200_E_INVALID, "triangle index out of range");
    if (nrm)
        for (int64_t i = 0; i < 3 * n_tri; ++i) {
            if ((int64_t)tri_nrm[i] >= n_nrm) return SetError(ctx, RTB200_E_INVALID, "normal index out of range");
            const float* n = nrm + 3 * (size_t)tri_nrm[i];
            if (!(std::isfinite(n[0]) && std::isfinite(n[1]) && std::isfinite(n[2])) ||
                !(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] > 0.0f))
                return SetError(ctx, RTB200_E_INVALID, "normals must be finite and nonzero");
        }
    s->meshes.push_back({(int64_t)s->tri_material.size(), n_tri, material, double_sided ? 1 : 0});
    const size_t base = s->tri9.size();
    s->tri9.resize(base + 9 * (size_t)n_tri);
    float* dst = s->tri9.data() + base;
    for (int64_t i = 0; i < n_tri; ++i)
        for (int j = 0; j < 3; ++j)
            std::memcpy(dst + 9 * i + 3 * j, xyz + 3 * (size_t)tri[3 * i + j], 12);
    s->tri_material.insert(s->tri_material.end(), (size_t)n_tri, material);
    s->tri_double_sided.insert(s->tri_double_sided.end(), (size_t)n_tri, (uint8_t)(double_sided ? 1 : 0));
    if (nrm || !s->tri_nrm9.empty()) {
        s->tri_nrm9.resize(s->tri9.size(), 0.0f);
        s->tri_smooth.resize(s->tri_material.size(), 0);
    }
    if (nrm) {
        float* nd = s->tri_nrm9.data() + base;
        for (int64_t i = 0; i < n_tri; ++i)
            for (int j = 0; j < 3; ++j)
                std::memcpy(nd + 9 * i + 3 * j, nrm + 3 * (size_t)tri_nrm[3 * i + j], 12);
        std::fill(s->tri_smooth.end() - n_tri, s->tri_smooth.end(), (uint8_t)1);
    }
    return RTB200_OK;
}

int rtb200_scene_add_mesh(rtb200_scene* s, const float* xyz, int64_t n_verts, const uint32_t* tri,
                          int64_t n_tri, int32_t material, int32_t double_sided)
{
    if (!s) return RTB200_E_INVALID;
    return AddMesh(s, xyz, n_verts, tri, n_tri, nullptr, 0, nullptr, material, double_sided);
}

int rtb200_scene_add_mesh_normals(rtb200_scene* s, const float* xyz, int64_t n_verts, const uint32_t* tri,
                                  int64_t n_tri, const float* normals, int64_t n_normals, const uint32_t* tri_normals,
                                  int32_t material, int32_t double_sided)
{
    if (!s) return RTB200_E_INVALID;
    if (!normals) return SetError(s->ctx, RTB200_E_INVALID, "no normals given");
    return AddMesh(s, xyz, n_verts, tri, n_tri, normals, n_normals, tri_normals, material, double_sided);
}

int rtb200_scene_add_risemesh(rtb200_scene* s, const rtb200_risemesh* m, int32_t material, int32_t use_cached_bvh)
{
    if (!s || !m) return RTB200_E_INVALID;
    std::vector<float> xyz;
    std::vector<uint32_t> tri;
    RisemeshTriangles(m, xyz, tri);
    const std::vector<uint32_t>* prims = nullptr;
    const std::vector<Node2>* nodes = use_cached_bvh ? RisemeshBvh(m, &prims) : nullptr;
    if (nodes && !ValidBVH2(*nodes, prims->size()))
        return SetError(s->ctx, RTB200_E_INVALID, "the mesh's cached BVH is malformed");
    std::vector<float> nrm;
    std::vector<uint32_t> tri_nrm;
    const bool smooth = RisemeshNormals(m, nrm, tri_nrm);
    const int rc = smooth ? rtb200_scene_add_mesh_normals(s, xyz.data(), (int64_t)(xyz.size() / 3), tri.data(),
                                                          (int64_t)(tri.size() / 3), nrm.data(),
                                                          (int64_t)(nrm.size() / 3), tri_nrm.data(), material,
                                                          RisemeshDoubleSided(m) ? 1 : 0)
                          : rtb200_scene_add_mesh(s, xyz.data(), (int64_t)(xyz.size() / 3), tri.data(),
                                                  (int64_t)(tri.size() / 3), material, RisemeshDoubleSided(m) ? 1 : 0);
    if (rc || !nodes || tri.empty()) return rc;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    rtb200_scene::Mesh& mesh = s->meshes.back();
    mesh.cached = true;
    mesh.cache_nodes = *nodes;
    mesh.cache_prims = *prims;
    return RTB200_OK;
}

namespace {
// The scene BVH: one reference build over all triangles, or, when a mesh
// brings its own BVH2, the two-level merge of per-mesh trees.
void BuildSceneBVH(rtb200_scene* s)
{
    bool any = false;
    for (const auto& m : s->meshes) any = any || m.cached;
    if (!any) {
        BuildReferenceBVH(s->tri9.data(), (int64_t)s->tri_material.size(), 0, s->bvh);
        return;
    }
    std::vector<BuiltBVH> own(s->meshes.size());
    std::vector<MeshBVH2> parts;
    for (size_t i = 0; i < s->meshes.size(); ++i) {
        const auto& m = s->meshes[i];
        if (m.count == 0) continue;
        if (m.cached) {
            parts.push_back({&m.cache_nodes, &m.cache_prims, m.first});
        } else {
            BuildReferenceBVH(s->tri9.data() + 9 * m.first, m.count, 0, own[i]);
            parts.push_back({&own[i].nodes2, &own[i].prims, m.first});
        }
    }
    MergeMeshBVHs(parts, s->bvh);
}
}  // namespace

int rtb200_scene_commit(rtb200_scene* s, int32_t layout)
{
    if (!s) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (s->committed) return SetError(ctx, RTB200_E_INVALID, "scene already committed");
    if (layout != RTB200_BVH_F32 && layout != RTB200_BVH_Q8 && layout != RTB200_BVH_W8 && layout != RTB200_BVH_F16)
        return SetError(ctx, RTB200_E_INVALID, "unknown BVH layout");
    const int64_t n_tri = (int64_t)s->tri_material.size();
    if (n_tri == 0) return SetError(ctx, RTB200_E_INVALID, "scene has no triangles");
    cudaSetDevice(ctx->device);
    const auto t0 = std::chrono::steady_clock::now();
    BuildSceneBVH(s);
    s->stack_bound = TraceStackBound(s->bvh);
    if (s->stack_bound > kTraceStackMax)
        return SetError(ctx, RTB200_E_INVALID, "BVH deeper than the traversal stack (" +
                        std::to_string(s->stack_bound) + " > " + std::to_string(kTraceStackMax) + " entries)");
    std::vector<GpuTri> tris;
    std::vector<GpuNode4> nf;
    std::vector<QNode4> nq;
    std::vector<HNode4> nh;
    std::vector<WNode8> nw;
    const void* nodes_src;
    size_t nodes_bytes;
    int64_t n_nodes = (int64_t)s->bvh.nodes4.size();
    if (layout == RTB200_BVH_W8) {
        int depth = 0;
        if (!EncodeWideNodes(s->bvh, nw, s->leaf_prims, depth))
            return SetError(ctx, RTB200_E_INVALID, "a BVH leaf holds more than 24 triangles");
        // One stack entry per node level below the root.
        if (depth - 1 > kW8MaxLevels)
            return SetError(ctx, RTB200_E_INVALID, "BVH deeper than the eight-wide traversal stack (" +
                            std::to_string(depth - 1) + " > " + std::to_string(kW8MaxLevels) + " levels)");
        EncodeWideTriangles(s->tri9.data(), s->leaf_prims, tris);
        nodes_src = nw.data();
        nodes_bytes = nw.size() * sizeof(WNode8);
        n_nodes = (int64_t)nw.size();
    } else {
        s->leaf_prims = s->bvh.prims;
        EncodeTriangles(s->tri9.data(), s->bvh, tris);
    }
    if (layout == RTB200_BVH_W8) {
    } else if (layout == RTB200_BVH_Q8) {
        EncodeQuantNodes(s->bvh, nq);
        nodes_src = nq.data();
        nodes_bytes = nq.size() * sizeof(QNode4);
    } else if (layout == RTB200_BVH_F16) {
        EncodeHalfNodes(s->bvh, nh);
        nodes_src = nh.data();
        nodes_bytes = nh.size() * sizeof(HNode4);
    } else {
        EncodeGpuNodes(s->bvh, nf);
        nodes_src = nf.data();
        nodes_bytes = nf.size() * sizeof(GpuNode4);
    }
    s->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    void* dn = nullptr;
    void* dt = nullptr;
    int rc = DevAlloc(ctx, &dn, nodes_bytes);
    if (rc) return rc;
    rc = DevAlloc(ctx, &dt, tris.size() * sizeof(GpuTri));
    if (rc) { DevFree(ctx, dn, nodes_bytes); return rc; }
    cudaError_t e = cudaMemcpyAsync(dn, nodes_src, nodes_bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, tris.data(), tris.size() * sizeof(GpuTri), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        DevFree(ctx, dn, nodes_bytes);
        DevFree(ctx, dt, tris.size() * sizeof(GpuTri));
        return CudaCheck(ctx, e, "scene upload");
    }
    s->d_nodes = dn;
    s->nodes_bytes = nodes_bytes;
    s->d_tris = (GpuTri*)dt;
    s->tris_bytes = tris.size() * sizeof(GpuTri);
    s->n_nodes = n_nodes;
    s->layout = layout;
    rc = UploadShading(s);
    if (rc) {
        DevFree(ctx, s->d_nodes, s->nodes_bytes);
        DevFree(ctx, s->d_tris, s->tris_bytes);
        s->d_nodes = nullptr;
        s->d_tris = nullptr;
        return rc;
    }
    s->committed = true;
    return RTB200_OK;
}

int rtb200_scene_info(const rtb200_scene* s, int64_t* n_tri, int64_t* n_nodes, int64_t* device_bytes,
                      double* build_seconds)
{
    if (!s) return RTB200_E_INVALID;
    if (n_tri) *n_tri = (int64_t)s->tri_material.size();
    if (n_nodes) *n_nodes = s->n_nodes;
    if (device_bytes) *device_bytes = (int64_t)(s->nodes_bytes + s->tris_bytes);
    if (build_seconds) *build_seconds = s->build_seconds;
    return RTB200_OK;
}

int rtb200_scene_destroy(rtb200_scene* s)
{
    if (!s) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    DevFree(ctx, s->d_nodes, s->nodes_bytes);
    DevFree(ctx, s->d_tris, s->tris_bytes);
    DevFree(ctx, s->d_in, s->stage_in);
    DevFree(ctx, s->d_out, s->stage_out);
    DevFree(ctx, s->d_counter, 256);
    FreeShading(s);
    delete s;
    return RTB200_OK;
}

struct rtb200_bvh_host {
    BuiltBVH b;
};

int rtb200_bvh_host_build(const float* tri9, int64_t n_tri, int32_t threads, rtb200_bvh_host** out)
{
    if (!out || n_tri < 0 || (n_tri > 0 && !tri9) || n_tri > (int64_t)UINT32_MAX) return RTB200_E_INVALID;
    rtb200_bvh_host* h = new (std::nothrow) rtb200_bvh_host();
    if (!h) return RTB200_E_OOM;
    BuildReferenceBVH(tri9, n_tri, threads, h->b);
    *out = h;
    return RTB200_OK;
}

int rtb200_bvh_host_from_risemesh(const rtb200_risemesh* m, int32_t use_cached_bvh, rtb200_bvh_host** out)
{
    if (!m || !out) return RTB200_E_INVALID;
    std::vector<float> xyz;
    std::vector<uint32_t> tri;
    RisemeshTriangles(m, xyz, tri);
    const std::vector<uint32_t>* prims = nullptr;
    const std::vector<Node2>* nodes = use_cached_bvh ? RisemeshBvh(m, &prims) : nullptr;
    if (nodes && !ValidBVH2(*nodes, prims->size())) return RTB200_E_INVALID;
    rtb200_bvh_host* h = new (std::nothrow) rtb200_bvh_host();
    if (!h) return RTB200_E_OOM;
    if (nodes) {
        MergeMeshBVHs({MeshBVH2{nodes, prims, 0}}, h->b);
    } else {
        std::vector<float> tri9(9 * (tri.size() / 3));
        for (size_t i = 0; i < tri.size(); ++i) std::memcpy(&tri9[3 * i], &xyz[3 * (size_t)tri[i]], 12);
        BuildReferenceBVH(tri9.data(), (int64_t)(tri.size() / 3), 0, h->b);
    }
    *out = h;
    return RTB200_OK;
}

int rtb200_bvh_host_info(const rtb200_bvh_host* h, int64_t* n2, int64_t* n4)
{
    if (!h) return RTB200_E_INVALID;
    if (n2) *n2 = (int64_t)h->b.nodes2.size();
    if (n4) *n4 = (int64_t)h->b.nodes4.size();
    return RTB200_OK;
}

int rtb200_bvh_host_export(const rtb200_bvh_host* h, void* nodes2, uint32_t* prims, void* nodes4)
{
    if (!h) return RTB200_E_INVALID;
    if (nodes2 && !h->b.nodes2.empty()) std::memcpy(nodes2, h->b.nodes2.data(), h->b.nodes2.size() * sizeof(Node2));
    if (prims && !h->b.prims.empty()) std::memcpy(prims, h->b.prims.data(), h->b.prims.size() * 4);
    if (nodes4 && !h->b.nodes4.empty()) std::memcpy(nodes4, h->b.nodes4.data(), h->b.nodes4.size() * sizeof(Node4));
    return RTB200_OK;
}

int rtb200_bvh_host_destroy(rtb200_bvh_host* h)
{
    if (!h) return RTB200_E_INVALID;
    delete h;
    return RTB200_OK;
}

int rtb200_cast_closest_device(rtb200_scene* s, const rtb200_ray* d_rays, int64_t n, rtb200_hit* d_hits,
                               void* stream)
{
    if (!s) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!s->committed) return SetError(ctx, RTB200_E_INVALID, "scene not committed");
    if (n < 0 || (n > 0 && (!d_rays || !d_hits))) return SetError(ctx, RTB200_E_INVALID, "bad ray buffers");
    if (!Aligned16(d_rays) || !Aligned16(d_hits)) return SetError(ctx, RTB200_E_INVALID, "ray/hit buffers must be 16-byte aligned");
    cudaSetDevice(ctx->device);
    return CudaCheck(ctx, LaunchCastClosest(s, d_rays, n, d_hits, (cudaStream_t)stream),
                     "closest-hit launch");
}

int rtb200_cast_any_device(rtb200_scene* s, const rtb200_ray* d_rays, int64_t n, uint8_t* d_occ, void* stream)
{
    if (!s) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!s->committed) return SetError(ctx, RTB200_E_INVALID, "scene not committed");
    if (n < 0 || (n > 0 && (!d_rays || !d_occ))) return SetError(ctx, RTB200_E_INVALID, "bad ray buffers");
    if (!Aligned16(d_rays)) return SetError(ctx, RTB200_E_INVALID, "ray buffer must be 16-byte aligned");
    cudaSetDevice(ctx->device);
    return CudaCheck(ctx, LaunchCastAny(s, d_rays, n, d_occ, (cudaStream_t)stream),
                     "any-hit launch");
}

int rtb200_scene_device_status(rtb200_scene* s, void* stream)
{
    if (!s) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!s->committed) return SetError(ctx, RTB200_E_INVALID, "scene not committed");
    cudaSetDevice(ctx->device);
    return CheckErrWord(s, (cudaStream_t)stream);
}

int rtb200_cast_closest(rtb200_scene* s, const rtb200_ray* rays, int64_t n, rtb200_hit* hits)
{
    if (!s) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!s->committed) return SetError(ctx, RTB200_E_INVALID, "scene not committed");
    if (n < 0 || (n > 0 && (!rays || !hits))) return SetError(ctx, RTB200_E_INVALID, "bad ray buffers");
    if (n == 0) return RTB200_OK;
    cudaSetDevice(ctx->device);
    int rc = RTB200_OK;
    const cudaError_t e = PipelinedCast(s, rays, n, hits, sizeof(rtb200_hit), rc,
        [s](const rtb200_ray* in, int64_t m, char* out, unsigned long long* counter, cudaStream_t st) {
            return LaunchCastClosestScratch(s, in, m, (rtb200_hit*)out, counter, s->d_err, st);
        });
    if (rc) return rc;
    if (e != cudaSuccess) return CudaCheck(ctx, e, "closest-hit cast");
    return CheckErrWord(s, ctx->stream);
}

int rtb200_cast_any(rtb200_scene* s, const rtb200_ray* rays, int64_t n, uint8_t* occ)
{
    if (!s) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!s->committed) return SetError(ctx, RTB200_E_INVALID, "scene not committed");
    if (n < 0 || (n > 0 && (!rays || !occ))) return SetError(ctx, RTB200_E_INVALID, "bad ray buffers");
    if (n == 0) return RTB200_OK;
    cudaSetDevice(ctx->device);
    int rc = RTB200_OK;
    const cudaError_t e = PipelinedCast(s, rays, n, occ, 1, rc,
        [s](const rtb200_ray* in, int64_t m, char* out, unsigned long long* counter, cudaStream_t st) {
            return LaunchCastAnyScratch(s, in, m, (uint8_t*)out, counter, s->d_err, st);
        });
    if (rc) return rc;
    if (e != cudaSuccess) return CudaCheck(ctx, e, "any-hit cast");
    return CheckErrWord(s, ctx->stream);
}

}  // extern "C"
