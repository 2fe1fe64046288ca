// pt_types.h -- device-side scene, job and queue descriptors of the spectral
// path tracer (pathtrace.cu), shared with the host code that fills them.
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "bvh_build.h"

#define RTB_HD __host__ __device__ __forceinline__

namespace rtb200 {

// Material models on the path (reference classes in src/Library/Materials/).
enum PtMatType : int {
    kMatLambertian = 0,   // LambertianSPF/LambertianBRDF
    kMatGGX = 1,          // GGXSPF/GGXBRDF, conductor Fresnel
    kMatDielectric = 2,   // DielectricSPF (no BSDF: per-wavelength path)
};

struct PtMaterial {
    int type;
    int refl;        // reflectance spectrum (Lambertian albedo); -1 = black
    int emit;        // emitted radiance spectrum; -1 = not an emitter
    int eta;         // conductor eta spectrum (GGX) or -1
    int kappa;       // conductor k spectrum (GGX) or -1
    float alpha;     // GGX roughness (alpha)
    float ior;       // dielectric index of refraction
    int pad;
};

// One luminary: a mesh whose material emits.  Points are drawn uniformly by
// area over its triangles (area CDF), like the reference's
// TriangleMeshGeometryIndexed::UniformRandomPoint.
struct PtLight {
    int first;       // first entry in the light-triangle array
    int count;
    float area;      // total area of the luminary
    float pdf;       // selection probability by power
    int emit;        // emitted radiance spectrum
    int bvh_pos;     // leaf position in the light BVH's order
    int kind;        // 0: a mesh luminary; 1: a point light at pos, radiance-like `le`
    float le;        // point light: luminance of colour x power (flat over wavelength)
    float pos[3];
    int mesh;        // the luminary's mesh (-1 for a point light)
};

// Light BVH node (LightBVHNode, Lights/LightBVH.h:100-115), preorder: the
// left child follows its parent, `right` is the right child's index.  A leaf
// (count 1) holds luminary `light`; `start` is the subtree's first leaf
// position.  Luminaries emit over the full sphere, so no cone is stored.
struct PtLightNode {
    float lo[3], hi[3];
    float power;
    int right;
    int light;
    int count;
    int start;
    int pad;
};

// Alias table over the luminaries for selection by power (Walker's alias
// method, built with Vose's algorithm: Utilities/AliasTable.h): entry i keeps
// i with probability prob, else gives alias.
struct PtLightAlias {
    float prob;
    int alias;
};

struct PtLightTri {
    float v0[3];
    float e1[3];
    float e2[3];
    float cdf;       // cumulative area fraction up to and including this triangle
    float pad[2];
};

struct PtCamera {
    float pos[3];
    float fwd[3];
    float right[3];  // scaled by tan(fov/2) * aspect
    float up[3];     // scaled by tan(fov/2)
    int width, height;
};

struct PtSettings {
    float lmin, lmax;        // wavelength range (nm)
    float ynorm;             // (lmax - lmin) / integral of y-bar over the range
    int max_depth;
    int rr_min_depth;
    float rr_threshold;
    int nee_per_lambda;      // 1: one light sample per wavelength (reference); 0: shared
    unsigned seed;
    int env;                 // uniform-sky radiance spectrum, -1 = none
    int env_visible;         // sky seen directly by camera rays
    int n_lights;
    int n_spectra;
    int filter;              // kFilterBox / kFilterSplat / kFilterWarp
    float filt_half;         // support half-width in pixels
    float filt_inv2s2;       // 1 / (2 sigma^2)
    float filt_norm;         // 1 / (2 pi sigma^2)
    float filt_sigma;        // Gaussian sigma in pixels (warp mode)
    float filt_trunc;        // exp(-K^2 / 2), K = half-width / sigma (warp mode)
    int light_bvh;           // pick NEE luminaries with the light BVH (when the scene has one)
    int sampler;             // kSamplerHash / kSamplerSobol / kSamplerSobolShuffled
    int max_bounce[3];       // diffuse, glossy, transmission scatters a path may take (255 = no limit)
    int single;              // 1: one wavelength per path (IntegrateRayNM); 0: hero + 3 companions
    int num_wl;              // single: wavelength bins (0 = continuous)
    float wl_step;           // single: (lmax - lmin) / num_wl
    float inv_spectral;      // 1 / paths per pixel sample (nSpectralSamples)
};

constexpr int kSamplerHash = 0;
constexpr int kSamplerSobol = 1;
constexpr int kSamplerSobolShuffled = 2;

// Bounce types (ScatteredRay::ScatRayType): the counters live in aux.w, one
// byte each.
constexpr int kBounceDiffuse = 0;
constexpr int kBounceGlossy = 1;
constexpr int kBounceTransmission = 2;

// Film modes of PtSettings::filter.  The reference splats into a filtered
// film only when the filter's half-support exceeds 0.501 pixel
// (PixelBasedRasterizerHelper.cpp:143-149); a narrower Gaussian instead warps
// the camera sample by the truncated kernel and averages with weight 1
// (PathTracingSpectralRasterizer.cpp:321-331, GaussianPixelFilter.h:109-127).
constexpr int kFilterBox = 0;     // uniform jitter in the pixel, 3-channel mean
constexpr int kFilterSplat = 1;   // Gaussian splat, 4 channels (XYZ and weight)
constexpr int kFilterWarp = 2;    // Gaussian-warped position, 3-channel mean

// Per-triangle shading attributes in leaf order: material | double-sided
// bit (bit 30), and the luminary index, or ~mesh for a triangle of a mesh
// that is no luminary (the index-of-refraction stack keys on meshes, the
// reference's objects; a luminary's mesh is PtLight::mesh).
struct PtTriAttr {
    int mat;
    int light;
};

// Index-of-refraction stack depth kept per path (PtPaths::media): dielectric
// meshes a path can be inside at once.  The reference's stack is unbounded;
// a path that would enter a fifth nested dielectric ends there.
constexpr int kPtMediaDepth = 4;

constexpr int kAttrDoubleSided = 1 << 30;
constexpr int kAttrSmooth = 1 << 29;   // interpolated vertex normals (PtScene::tri_normals)
constexpr int kAttrMatMask = (1 << 24) - 1;

// Path flags (meta.z).
constexpr unsigned kFlagDepthMask = 0xffu;
constexpr unsigned kFlagConsiderEmission = 1u << 8;
constexpr unsigned kFlagFinishing = 1u << 9;
constexpr unsigned kFlagSpecular = 1u << 10;
constexpr unsigned kFlagInMedium = 1u << 11;   // PtPaths::media holds at least one mesh
constexpr unsigned kTermShift = 12;        // 4 bits: terminated wavelengths

// Shadow-ray queue entry, 48 bytes.
struct ShadowEntry {
    float4 o;        // origin, w = tmax
    float4 d;        // direction, w = path slot (int bits)
    float4 c;        // contribution per wavelength (added when unoccluded)
};

// Counters in device memory.
enum PtCounter : int {
    kCntActive = 0,     // paths to extend this iteration
    kCntActiveNext = 1,
    kCntFree = 2,       // finished / empty slots to regenerate
    kCntFreeNext = 3,
    kCntShadow = 4,
    kCntSegments = 5,   // extended rays (statistics)
    kCntShadowRays = 6,
    kCntAssigned = 7,   // free slots given camera samples this iteration
    kCntClass = 8,      // kCntClass + c: active paths of shading class c (KClassify)
    kCntJobs = 11,      // entries of the job id list (written by the host)
    kCntCount = 16,
};

struct PtEnvMap;   // env_map.h

struct PtScene {
    const void* nodes;
    int layout;
    int n_nodes;
    const GpuTri* tris;
    int ntri;
    const PtTriAttr* attr;
    const PtMaterial* mats;
    const float* spectra;      // spectrum table: float4 header per id, then samples (Spec)
    const PtLight* lights;
    const PtLightTri* light_tris;
    const PtLightNode* light_nodes;   // light BVH (null with fewer than two luminaries)
    const PtLightAlias* light_alias;  // alias table over the luminaries (power selection)
    // Vertex normals of triangles marked kAttrSmooth, in leaf order: x, y, z
    // hold the three vertices' unit normals octahedron-encoded (two signed
    // 16-bit components each, OctDecode in pt_device.cuh); null when no mesh
    // of the scene has normals.
    const uint4* tri_normals;
    // Image environment (env_map.h), or null: then PtSettings::env names a
    // uniform sky's spectrum, or none.
    const PtEnvMap* env_map;
    // Material of each mesh, for the indices of the meshes on a path's
    // index-of-refraction stack.
    const int* mesh_mat;
};

// Octahedral encoding of a unit vector (Cigolle et al., "A Survey of
// Efficient Representations for Independent Unit Vectors", JCGT 3(2), 2014):
// project onto the octahedron |x| + |y| + |z| = 1, fold the lower half over
// the upper, keep (x, y) as signed 16-bit fractions.  FP32 throughout so
// host and restatement encode bit for bit.
RTB_HD unsigned OctEncode(float x, float y, float z)
{
    const float s = fabsf(x) + fabsf(y) + fabsf(z);
    float u = s > 0.0f ? x / s : 0.0f, v = s > 0.0f ? y / s : 0.0f;
    if (z < 0.0f) {
        const float fu = (1.0f - fabsf(v)) * (u >= 0.0f ? 1.0f : -1.0f);
        const float fv = (1.0f - fabsf(u)) * (v >= 0.0f ? 1.0f : -1.0f);
        u = fu;
        v = fv;
    }
    const int qu = (int)rintf(fminf(fmaxf(u, -1.0f), 1.0f) * 32767.0f);
    const int qv = (int)rintf(fminf(fmaxf(v, -1.0f), 1.0f) * 32767.0f);
    return ((unsigned)qu & 0xffffu) | ((unsigned)qv << 16);
}

struct PtPaths {
    float4* ray_o;   // origin, tmin
    float4* ray_d;   // direction, tmax
    float4* hit;     // t, leaf slot (int bits, -1 miss), a, b
    float4* thr;     // throughput per wavelength
    float4* L;       // radiance per wavelength
    float4* aux;     // x hero wavelength, y bsdf pdf
    uint4* meta;     // x pixel, y sample, z flags, w rng key
    // Index-of-refraction stack (Utilities/IORStack.h): the dielectric
    // meshes the path is inside, innermost last, -1 past the top; read only
    // when meta.z has kFlagInMedium (an empty stack otherwise).
    int4* media;
};

constexpr int kPtMaxJobs = 1024;   // jobs per engine (one KAssign thread each)

// Camera samples handed to one job in one iteration: free-queue entries
// [off, next job's off) take the job's samples base, base + 1, ...
struct PtAssign {
    unsigned long long base;
    int off;
    int jid;
};

struct PtQueues {
    int* active;        // current
    int* active_next;
    int* free_;         // current
    int* free_next;
    ShadowEntry* shadow;
    int* cnt;           // PtCounter
    unsigned long long* sample_ctr;
    unsigned long long* trace_ctr;   // [2]: extend, connect
    unsigned* err;
    PtAssign* assign;                // [max jobs], written by KAssign
    int* shade;                      // [kShadeClasses][capacity]: active slots by shading class
    int capacity;
};

// Shading classes: paths that escaped or hit Lambertian surfaces, GGX
// conductors, smooth dielectrics.  KShade runs them as contiguous ranges so a
// warp shades one material model.
constexpr int kShadeClasses = 3;

struct PtFilm {
    float* pass;        // 3 floats per pixel, atomically accumulated this call
    float* sum;         // 3 floats per pixel, compensated running sum
    float* comp;        // 3 floats per pixel, Kahan compensation
};

// One image being rendered: its scene, camera, settings, film and sample
// counters.  The engine's kernels read a table of these; every path slot
// records which job it belongs to (aux.z).
struct PtJobDev {
    PtScene scene;
    PtCamera cam;
    PtSettings set;
    int npix;                          // pixels this request samples (adaptive: unconverged ones)
    int pad;
    const unsigned* px_list;           // adaptive: the pixels sampled, else null (all pixels in order)
    double* lum;                       // adaptive: per pixel sum of Y and of Y^2 over its samples, else null
    float* film;                       // 3 (box, warp) or 4 (splat) floats per pixel, this request's samples
    unsigned long long sample_begin;   // first sample index (per pixel) of the request
    unsigned long long total;          // npix * spp of the request
    unsigned long long* sample_ctr;    // samples handed out so far (device)
    unsigned long long* done_ctr;      // samples finished and splatted (device)
};

}  // namespace rtb200
