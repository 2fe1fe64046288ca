// core.h -- internal context and scene state behind the C ABI (rtb200.h).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <unordered_map>
#include <string>
#include <vector>

#include "../../include/rtb200.h"
#include "bvh_build.h"
#include "pt_types.h"

struct rtb200_ctx {
    int device = 0;
    int num_sms = 0;
    size_t budget = 0;      // 0 = no cap
    size_t in_use = 0;
    cudaStream_t stream = nullptr;
    // Copy streams, a second trace stream and events of the pipelined
    // host-buffer casts.
    cudaStream_t copy_in = nullptr, copy_out = nullptr, trace2 = nullptr;
    cudaEvent_t ev_up[2] = {}, ev_trace[2] = {}, ev_down[2] = {};
    std::mutex mu;
    std::string err;
    // Freed blocks of DevFreeCached by size, for reuse in stream order on
    // `stream` (films come and go with every served request; cudaFree would
    // synchronise the device each time).  Not counted in in_use.
    std::unordered_map<size_t, std::vector<void*>> cache;
    size_t cached = 0;
};

struct rtb200_scene {
    rtb200_ctx* ctx = nullptr;
    // host geometry, scene-wide triangle numbering
    std::vector<float> tri9;
    std::vector<int32_t> tri_material;
    std::vector<uint8_t> tri_double_sided;
    // Vertex normals (9 floats per triangle, corner order) of meshes added
    // with normals; empty until the first such mesh, then as long as tri9.
    std::vector<float> tri_nrm9;
    std::vector<uint8_t> tri_smooth;
    struct Mesh {
        int64_t first, count;
        int32_t material;
        int32_t double_sided;
        // BVH2 read with the mesh (a .risemesh cache): mesh-local leaf order
        bool cached = false;
        std::vector<rtb200::Node2> cache_nodes;
        std::vector<uint32_t> cache_prims;
    };
    std::vector<Mesh> meshes;
    // spectral shading data
    std::vector<float> spectra;                 // 81 samples per spectrum (5 nm grid)
    // Binned packets (SpectralPacket): spectrum id -> begin, end, amplitudes;
    // `spectra` holds their values at the grid points for host-side use.
    struct Packet {
        int32_t id;
        float begin, end;
        std::vector<float> amps;
    };
    std::vector<Packet> packets;
    // RGB colours' sigmoid polynomials: spectrum id -> c0, c1, c2, scale.
    struct Sigmoid {
        int32_t id;
        float c[4];
    };
    std::vector<Sigmoid> sigmoids;
    // Black bodies: spectrum id -> temperature, scale.
    struct Blackbody {
        int32_t id;
        float t, scale;
    };
    std::vector<Blackbody> blackbodies;
    size_t spectra_table_bytes = 0;
    std::vector<rtb200::PtMaterial> materials;
    bool mixed_shading = false;      // materials of more than one shading class
    int shade_class = -1;            // otherwise the one class (RTB200_MAT_* type), set at commit
    int32_t env = -1, env_visible = 1;
    // Image environment (rtb200_scene_set_environment_map): RGB texels, the
    // world -> map rotation, radiance scale, importance-sampling tables.
    std::vector<float4> env_texels;
    int env_w = 0, env_h = 0;
    float env_rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    float env_scale = 1.0f;
    std::vector<float> env_marginal, env_conditional;
    void* d_env = nullptr;           // one block: PtEnvMap, texels, tables, uplift table
    size_t env_bytes = 0;
    std::vector<rtb200::PtLight> lights;        // built at commit
    std::vector<rtb200::PtLightTri> light_tris;
    // device copies (path tracer)
    rtb200::PtTriAttr* d_attr = nullptr;
    std::vector<int> mesh_mat;       // material per mesh, built at commit
    int* d_mesh_mat = nullptr;
    rtb200::PtMaterial* d_mats = nullptr;
    float* d_spectra = nullptr;
    rtb200::PtLight* d_lights = nullptr;
    rtb200::PtLightTri* d_light_tris = nullptr;
    std::vector<rtb200::PtLightNode> light_nodes;  // light BVH, built at commit
    struct PointLight {
        float pos[3], color[3], power;
    };
    std::vector<PointLight> point_lights;
    rtb200::PtLightNode* d_light_nodes = nullptr;
    std::vector<rtb200::PtLightAlias> light_alias;  // built at commit
    rtb200::PtLightAlias* d_light_alias = nullptr;
    std::vector<uint4> tri_normals;      // leaf order, built at commit (OctEncode)
    uint4* d_tri_normals = nullptr;
    size_t shade_bytes = 0;
    bool committed = false;
    int32_t layout = RTB200_BVH_F32;
    int64_t n_nodes = 0;
    int32_t stack_bound = 0;         // TraceStackBound of the committed BVH
    double build_seconds = 0.0;
    rtb200::BuiltBVH bvh;            // kept for the path tracer's emitter tables
    std::vector<uint32_t> leaf_prims;   // triangle order of d_tris (input index per slot)
    // device data
    void* d_nodes = nullptr;
    size_t nodes_bytes = 0;
    rtb200::GpuTri* d_tris = nullptr;
    size_t tris_bytes = 0;
    // per-scene scratch: work counter (u64) and error word (u32)
    unsigned long long* d_counter = nullptr;
    unsigned* d_err = nullptr;
    // staging for the host-buffer entry points
    void* d_in = nullptr;
    void* d_out = nullptr;
    size_t stage_in = 0, stage_out = 0;
};

namespace rtb200 {

// Device allocation against the context budget.
int DevAlloc(rtb200_ctx* ctx, void** p, size_t bytes);
void DevFree(rtb200_ctx* ctx, void* p, size_t bytes);
// The same for blocks used only by work on ctx->stream: a freed block is kept
// (up to kDevCacheBytes in all) and handed to the next request of the same
// size, which stream order makes safe.  DevReleaseCache returns them all.
constexpr size_t kDevCacheBytes = size_t(4) << 30;
int DevAllocCached(rtb200_ctx* ctx, void** p, size_t bytes);
void DevFreeCached(rtb200_ctx* ctx, void* p, size_t bytes);
void DevReleaseCache(rtb200_ctx* ctx);
int SetError(rtb200_ctx* ctx, int code, const std::string& msg);
// .risemesh accessors (risemesh.cpp).
bool RisemeshTriangles(const rtb200_risemesh* m, std::vector<float>& xyz, std::vector<uint32_t>& tri);
const std::vector<rtb200::Node2>* RisemeshBvh(const rtb200_risemesh* m, const std::vector<uint32_t>** prims);
bool RisemeshDoubleSided(const rtb200_risemesh* m);
bool RisemeshNormals(const rtb200_risemesh* m, std::vector<float>& nrm, std::vector<uint32_t>& tri_nrm);
// Image environments (envmap.cpp) and the RGB uplift table (rgb_uplift.cpp).
void EnvRotation(const double orient_rad[3], float rot[9]);
void BuildEnvTables(const std::vector<float4>& texels, int width, int height, float scale,
                    std::vector<float>& marginal, std::vector<float>& conditional);
const std::vector<float>& UpliftTable();

int CudaCheck(rtb200_ctx* ctx, cudaError_t e, const char* what);

// Shading tables of a committed scene (pt_api.cpp): per-triangle attributes
// in leaf order, materials, spectra, luminaries.
int UploadShading(rtb200_scene* s);
void FreeShading(rtb200_scene* s);

// Kernel launchers (raycast.cu).  Asynchronous on `stream`.
cudaError_t LaunchCastClosest(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                              rtb200_hit* d_hits, cudaStream_t stream);
cudaError_t LaunchCastAny(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                          uint8_t* d_occ, cudaStream_t stream);
// Closest-hit launch with caller-provided scratch (work counter and error
// word); clears nothing itself.
cudaError_t LaunchCastAnyScratch(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n, uint8_t* d_occ,
                                 unsigned long long* counter, unsigned* err, cudaStream_t stream);
cudaError_t LaunchCastClosestScratch(const rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                                     rtb200_hit* d_hits, unsigned long long* counter, unsigned* err,
                                     cudaStream_t stream);

}  // namespace rtb200
