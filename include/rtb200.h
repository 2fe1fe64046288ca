/* rtb200.h -- C ABI of the B200 spectral path tracer and BVH ray caster.
 *
 * A drop-in for one hot path of the RISE renderer: the unidirectional
 * hero-wavelength spectral path tracer driven by PixelBasedRasterizerHelper
 * and the BVH ray caster beneath it.  Plain pointers and sizes only; every
 * call returns an RTB200_* status code and never throws.  Device memory is
 * owned by the context.  A context is single-owner: calls on one context are
 * serialised by an internal mutex.
 *
 * Entry point -> reference interface it replaces (paths relative to the
 * reference source tree):
 *
 *   rtb200_ctx_create / _destroy
 *       the Job/RuntimeContext ownership of a render (Job.cpp:9268-9318)
 *   rtb200_scene_create / _add_mesh / _commit / _destroy
 *       TriangleMeshGeometryIndexed::DoneIndexedTriangles + the BVH
 *       constructor (Geometry/TriangleMeshGeometryIndexed.cpp:444-537,
 *       Acceleration/BVH.h:162-192) and ObjectManager::PrepareForRendering
 *       (Managers/ObjectManager.cpp:404)
 *   rtb200_cast_closest[_device]
 *       IRayCaster::CastRay's intersection step, i.e.
 *       ObjectManager::IntersectRay (Managers/ObjectManager.cpp:270-318) ->
 *       BVH::IntersectRay (Acceleration/BVH.h:1475-1560), batched
 *   rtb200_cast_any[_device]
 *       IRayCaster::CastShadowRay (Rendering/RayCaster.cpp:1958-1966) ->
 *       ObjectManager::IntersectShadowRay (Managers/ObjectManager.cpp:320-374)
 *       -> BVH::IntersectRay_IntersectionOnly (Acceleration/BVH.h:1639-1717),
 *       batched
 */
#ifndef RTB200_H
#define RTB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define RTB200_OK          0
#define RTB200_E_INVALID   1  /* bad argument or call order */
#define RTB200_E_OOM       2  /* device allocation failed */
#define RTB200_E_BUDGET    3  /* request exceeds the context's memory budget */
#define RTB200_E_TIMEOUT   4  /* a bounded device wait gave up */
#define RTB200_E_DEVICE    5  /* CUDA error or device-side error word set */
#define RTB200_E_NOT_READY 6  /* asynchronous work still in flight */
#define RTB200_E_CANCELLED 7  /* a progress callback stopped the render; the film
                                 holds the pixel samples completed */

/* BVH device layouts for rtb200_scene_commit. */
#define RTB200_BVH_F32     0  /* FP32 child boxes, 128-byte 4-wide nodes */
#define RTB200_BVH_Q8      1  /* 8-bit conservative child boxes, 64-byte nodes */
#define RTB200_BVH_W8      2  /* 8-wide nodes with 8-bit conservative child boxes, 80 bytes */
#define RTB200_BVH_F16     3  /* binary16 child boxes rounded outward, 64-byte nodes */

typedef struct rtb200_ctx rtb200_ctx;
typedef struct rtb200_scene rtb200_scene;

/* One ray, 32 bytes: origin, tmin, unit or non-unit direction, tmax.
 * Hits are reported for tmin < t < tmax (tmax may be +inf). */
typedef struct {
    float ox, oy, oz, tmin;
    float dx, dy, dz, tmax;
} rtb200_ray;

/* One closest-hit result, 16 bytes.  prim is the triangle index in the
 * order triangles were added to the scene (-1 on a miss); t is the
 * reference's double-precision distance rounded to FP32; (a, b) are the
 * barycentric weights of the triangle's second and third vertex. */
typedef struct {
    float t;
    int32_t prim;
    float a, b;
} rtb200_hit;

/* ---- context ----------------------------------------------------------- */

/* Create a context on CUDA device `device`.  budget_bytes caps the device
 * memory the context may hold (0 = no cap). */
int rtb200_ctx_create(int device, size_t budget_bytes, rtb200_ctx** out);
int rtb200_ctx_destroy(rtb200_ctx* ctx);
/* Message for the last failing call on this context ("" if none). */
const char* rtb200_last_error(const rtb200_ctx* ctx);
/* Device bytes currently held by the context. */
size_t rtb200_ctx_bytes_in_use(const rtb200_ctx* ctx);

/* ---- scenes ------------------------------------------------------------ */

int rtb200_scene_create(rtb200_ctx* ctx, rtb200_scene** out);
/* Add an indexed triangle mesh: xyz holds n_verts float triples, tri holds
 * n_tri uint32 index triples.  Triangles are numbered scene-wide in the
 * order they are added.  material is an index into the scene's material
 * table (ignored by the ray caster).  double_sided follows the reference's
 * bDoubleSided (normals face the incoming ray). */
int rtb200_scene_add_mesh(rtb200_scene* scene, const float* xyz, int64_t n_verts,
                          const uint32_t* tri, int64_t n_tri, int32_t material,
                          int32_t double_sided);
/* The same with vertex normals for shading (ITriangleMeshGeometryIndexed's
 * normal list and per-corner normal indices, IndexedTriangle::iNormals):
 * normals holds n_normals float triples, tri_normals n_tri index triples
 * into it.  The path tracer shades with the normal interpolated at the hit,
 * n0 + (n1 - n0) a + (n2 - n0) b normalised
 * (Geometry/TriangleMeshGeometryIndexedSpecializations.h:194-199,
 * Objects/Object.cpp:543), the face normal oriented to its side serving as
 * the geometric normal; a double-sided mesh turns each towards the incoming
 * ray (TriangleMeshGeometryIndexed.cpp:170-188).  Normals must be finite and
 * nonzero; they are stored unit length in a 32-bit octahedral encoding. */
int rtb200_scene_add_mesh_normals(rtb200_scene* scene, const float* xyz, int64_t n_verts,
                                  const uint32_t* tri, int64_t n_tri, const float* normals,
                                  int64_t n_normals, const uint32_t* tri_normals, int32_t material,
                                  int32_t double_sided);
/* Build the BVH on the host (all cores) and upload it.  layout is one of
 * RTB200_BVH_*.  Meshes cannot be added after commit.  The device traversal
 * stack holds at most 128 deferred nodes; a BVH whose worst root-to-node path
 * defers more (only deeply nested geometry does) is refused with
 * RTB200_E_INVALID, where the reference's unbounded stack
 * (Acceleration/BVH.h:1311-1320) would go on. */
int rtb200_scene_commit(rtb200_scene* scene, int32_t layout);
/* ---- .risemesh files ---------------------------------------------------- */

/* A parsed .risemesh (the reference's mesh file, versions 1 to 5:
 * TriangleMeshGeometryIndexed::Serialize / Deserialize,
 * Geometry/TriangleMeshGeometryIndexed.cpp:585-980), with the BVH2 cache its
 * v3+ files may carry (BVH::Serialize / Deserialize, Acceleration/BVH.h:338-423).
 * rtb200_risemesh_parse reads a file's bytes; RTB200_E_INVALID for a
 * malformed or truncated file, an index out of range, a cache whose leaf
 * order does not list every triangle, or a v1..v3 file that carries a legacy
 * BSP / octree block.  rtb200_risemesh_info: any output may
 * be NULL; n_bvh_nodes is 0 without a cache.
 *
 * rtb200_scene_add_risemesh adds the mesh's triangles (vertex positions
 * rounded to FP32; its own double-sided flag) and, unless the file marks the
 * mesh as shaded with face normals, its vertex normals for smooth shading
 * (as rtb200_scene_add_mesh_normals).  With use_cached_bvh and a
 * cache in the file, the cache is checked (child pairs after their parent
 * and in range, each node reached once, leaf ranges inside the leaf order,
 * depth <= 1024, ordered boxes; RTB200_E_INVALID otherwise) and the scene's
 * commit skips the SAH build of this mesh: a scene with a cached mesh is
 * built in two levels, a top level over the meshes' root boxes and below it
 * each mesh's own BVH2 (the cache, or the reference build of that mesh
 * alone), then collapsed to four-wide nodes as the reference's loader does
 * (BVH.h:414-418).  A scene of one cached mesh traverses the file's node
 * layout unchanged. */
typedef struct rtb200_risemesh rtb200_risemesh;
int rtb200_risemesh_parse(const void* bytes, size_t n_bytes, rtb200_risemesh** out);
int rtb200_risemesh_info(const rtb200_risemesh* mesh, int32_t* version, int64_t* n_points, int64_t* n_tri,
                         int32_t* double_sided, int64_t* n_bvh_nodes);
/* The mesh's triangles as 9 floats each (v0, v1, v2), FP32-rounded. */
int rtb200_risemesh_triangles(const rtb200_risemesh* mesh, float* tri9);
/* The vertex normals of each triangle's corners, 9 floats per triangle;
 * RTB200_E_INVALID when the mesh shades with face normals or has none. */
int rtb200_risemesh_normals(const rtb200_risemesh* mesh, float* nrm9);
int rtb200_risemesh_destroy(rtb200_risemesh* mesh);
int rtb200_scene_add_risemesh(rtb200_scene* scene, const rtb200_risemesh* mesh, int32_t material,
                              int32_t use_cached_bvh);

/* Node / triangle counts and device bytes of a committed scene. */
int rtb200_scene_info(const rtb200_scene* scene, int64_t* n_tri, int64_t* n_nodes,
                      int64_t* device_bytes, double* build_seconds);
int rtb200_scene_destroy(rtb200_scene* scene);

/* ---- spectral materials and lights ------------------------------------ */

/* Spectra are tabulated at 81 samples, 380..780 nm in 5 nm steps, linearly
 * interpolated (the reference's SPD interpolation, Utilities/Color/
 * ColorUtils.cpp:270-300); they stand in for the reference's spectral
 * painters (IPainter::GetColorNM, Interfaces/IPainter.h:67). */
#define RTB200_SPECTRUM_SAMPLES 81

/* Material models (reference classes under src/Library/Materials/). */
#define RTB200_MAT_LAMBERTIAN 0   /* LambertianSPF + LambertianBRDF */
#define RTB200_MAT_GGX        1   /* GGXSPF + GGXBRDF, conductor Fresnel */
#define RTB200_MAT_DIELECTRIC 2   /* DielectricSPF, no BSDF */

typedef struct {
    int32_t type;         /* RTB200_MAT_* */
    int32_t reflectance;  /* spectrum id: Lambertian albedo (-1 = black) */
    int32_t emission;     /* spectrum id of emitted radiance (-1 = none);
                             LambertianEmitter: one-sided, radiance = spectrum */
    int32_t eta, kappa;   /* GGX conductor spectra (-1 = unused); for a dielectric,
                             eta >= 0 names a spectrum holding its index of
                             refraction per wavelength (a dispersive IOR: the
                             reference's `ior` scalar painter evaluated by
                             IScalarPainter::GetValueAtNM), else `ior` holds */
    float alpha;          /* GGX roughness; for a dielectric, the Phong exponent of
                             its transmitted lobe (the reference's `scattering`,
                             DielectricSPF.cpp:248-272; 0 or >= 1e6: smooth) */
    float ior;            /* dielectric index of refraction (constant) */
} rtb200_material;

/* Returns the new spectrum / material id in *id_out.  Materials are
 * referenced by rtb200_scene_add_mesh's `material`; a mesh whose material
 * emits becomes one luminary (area light) at commit. */
int rtb200_scene_add_spectrum(rtb200_scene* scene, const float* values, int32_t* id_out);
int rtb200_scene_add_material(rtb200_scene* scene, const rtb200_material* m, int32_t* id_out);
/* A binned spectrum as the reference's spectral painters hold it
 * (SpectralPacket, Utilities/Color/SpectralPacket.h:80-100,285-297; made by
 * Job::AddSpectralColorPainter, Job.cpp:1557-1582): n amplitudes over
 * [lambda_begin, lambda_end]; the value at nm is the amplitude of the bin
 * holding it, 0 outside the range.  Shares the id space of
 * rtb200_scene_add_spectrum. */
int rtb200_scene_add_spectral_packet(rtb200_scene* scene, float lambda_begin, float lambda_end, int32_t n,
                                     const float* amplitudes, int32_t* id_out);

/* RGB colours as spectra, as the reference's RGB painters evaluate them
 * (UniformColorPainter::GetColorNM, Painters/UniformColorPainter.h:40-76):
 * the Jakob-Hanika sigmoid polynomial of the colour in linear Rec.709,
 * S(l) = scale * s(c0 t^2 + c1 t + c2), t = (l - 380) / 400, 0 outside
 * 380..780 nm, s(x) = 1/2 + x / (2 sqrt(1 + x^2)).  ALBEDO clamps the colour
 * to [0, 1] (scale 1; RGBAlbedoSpectrum, the reference painters' default);
 * UNBOUNDED divides it by its largest channel, which becomes the scale
 * (RGBUnboundedSpectrum).  rtb200_rgb_uplift writes (c0, c1, c2, scale) and
 * needs no device; its coefficient table is built on first use (a few seconds
 * on all host cores) by the reference's generator steps
 * (tools/JakobHanikaLUTGen.cpp, Rec.709, 64^3 cells per largest channel).
 * rtb200_rgb_uplift_table copies that table (3 * 64^3 cells of c0, c1, c2,
 * floats, ordered [largest channel][z][x][y]).  rtb200_scene_add_rgb_spectrum
 * adds such a spectrum to a scene's table (id space of
 * rtb200_scene_add_spectrum). */
#define RTB200_RGB_ALBEDO 0
#define RTB200_RGB_UNBOUNDED 1
int rtb200_rgb_uplift(const double* rgb, int32_t kind, double* coeffs_and_scale);
int rtb200_rgb_uplift_table(float* coeffs);
int rtb200_scene_add_rgb_spectrum(rtb200_scene* scene, const double* coeffs_and_scale, int32_t* id_out);
/* A black body of the given temperature (K): scale * Planck's function of the
 * wavelength in metres, divided by its value at 0.0029 / T m when normalize
 * is set (Job::AddBlackBodyPainter / BlackBodyPainter::GetColorNM,
 * Painters/BlackBodyPainter.cpp:26-43,103-106,152-170).  Same id space. */
int rtb200_scene_add_blackbody(rtb200_scene* scene, double temperature, double scale, int32_t normalize,
                               int32_t* id_out);
/* A point light (omni_light: Job::AddPointOmniLight, Lights/PointLight.h:49-57):
 * next-event estimation gives it the luminance of colour x power at every
 * wavelength, times cos / distance^2 (LightSampler.cpp:2097-2130); it joins
 * the luminaries in light selection with weight max(colour) x power x 4 pi
 * (its radiant exitance) and cannot be hit by rays. */
int rtb200_scene_add_point_light(rtb200_scene* scene, const float* position, const float* color, float power);
/* Uniform sky: radiance spectrum for rays that escape (-1 = none); visible
 * selects whether camera rays see it directly. */
int rtb200_scene_set_environment(rtb200_scene* scene, int32_t spectrum, int32_t visible);

/* Image environment: the rasterizer's radiance_map bound to an HDR texture
 * painter (RadianceMapConfig, Utilities/RadianceMapConfig.h; RadianceMap,
 * Rendering/RadianceMap.h; Job::AddHDRTexturePainter, Job.cpp:2216-2265).
 * rgb: width x height linear Rec.709 texels, rows top to bottom, as the
 * reference's HDR reader delivers them (rtb200_hdr_decode).  A world
 * direction is rotated by the Euler angles orientation_deg (x, y, z in
 * degrees, radiance_orient; null = none), mapped to the light-probe (angular)
 * image, read with the bilinear filter at the base level, uplifted to a
 * spectrum per lookup (RGBUnboundedSpectrum) and scaled by `scale`
 * (radiance_scale).  Next-event estimation draws directions from the
 * reference's 64 x 64 importance table (EnvironmentSampler) with
 * power-heuristic MIS against BSDF sampling.  visible: camera rays see the
 * map (radiance_background).  Replaces a uniform sky and vice versa. */
int rtb200_scene_set_environment_map(rtb200_scene* scene, const float* rgb, int32_t width, int32_t height,
                                     float scale, const float* orientation_deg, int32_t visible);
/* Replaces the image environment's rotation by a world -> map matrix
 * (row major, map_i = sum_j rot9[3 i + j] world_j): a host holding the
 * radiance map's transform (RadianceMap::GetTransform) passes it as is. */
int rtb200_scene_set_environment_rotation(rtb200_scene* scene, const float* rot9);

/* Decodes a Radiance HDR (RGBE) file held in memory as the reference's
 * HDRReader does (RasterImages/HDRReader.cpp): *width, *height, and with rgb
 * non-null width x height x 3 floats, rows top to bottom. */
int rtb200_hdr_decode(const uint8_t* bytes, int64_t n, int32_t* width, int32_t* height, float* rgb);

/* ---- render jobs (the rasterizer) -------------------------------------- */

/* Settings of one progressive render.  Replaces the parameters of
 * RISE_API_CreatePathTracingSpectralRasterizer (RISE_API.h:3112-3141) and the
 * pinhole camera (Cameras/PinholeCamera.cpp:182-217) for this path. */
typedef struct {
    int32_t width, height;
    float cam_pos[3], cam_look[3], cam_up[3];
    float fov_deg;            /* vertical field of view */
    float lambda_min, lambda_max;
    int32_t max_depth;        /* path vertices, as the reference's max depth */
    int32_t rr_min_depth;     /* Russian roulette from this depth (reference: 3) */
    float rr_threshold;       /* reference: 0.05 */
    int32_t nee_per_lambda;   /* 1: one light sample per wavelength, as the
                                 reference; 0: one shared sample per vertex */
    uint32_t seed;
    int32_t max_paths;        /* path-pool capacity (0 = automatic) */
    int32_t filter;           /* RTB200_FILTER_* */
    float filter_size;        /* Gaussian: kernel width in pixels (support = size / 2), 0 < size <= 16 */
    float filter_sigma;       /* Gaussian: standard deviation in pixels, > 0 */
    int32_t adaptive_max_spp; /* adaptive sampling: maximum samples per pixel (0 = off) */
    float adaptive_threshold; /* adaptive sampling: relative standard error to converge (reference: 0.01) */
    int32_t light_selection;  /* RTB200_LIGHTS_* */
    int32_t sampler;          /* RTB200_SAMPLER_* */
    /* Per-type bounce limits (StabilityConfig::maxDiffuseBounce /
     * maxGlossyBounce / maxTransmissionBounce, PathTransportUtilities.h:170-221):
     * when bounce_limits is set, a path ends once a scatter of a type would
     * make that type's count exceed its limit (diffuse: Lambertian and the GGX
     * multiple-scattering lobe; glossy: GGX specular and dielectric
     * reflection; transmission: dielectric refraction).  max_depth still caps
     * the number of path vertices (the reference's default is 128). */
    int32_t bounce_limits;
    int32_t max_diffuse_bounce, max_glossy_bounce, max_transmission_bounce;
    /* Wavelength sampling (SpectralConfig, Utilities/SpectralConfig.h;
     * PathTracingSpectralRasterizer::IntegratePixelSpectral,
     * Rendering/PathTracingSpectralRasterizer.cpp:121-198).
     * RTB200_SPECTRAL_HWSS: four wavelengths per path, a quarter of the range
     * apart (the reference's `hwss true`).  At a dielectric whose index of
     * refraction differs between the hero and a companion wavelength, the
     * companions end and the hero continues alone, its sample counted as one
     * wavelength (SampledWavelengths::TerminateSecondary; the reference instead
     * continues each wavelength on its own single-wavelength path from there,
     * PathTracingIntegrator.cpp:4336-4365 — the same expectation).
     * RTB200_SPECTRAL_SINGLE: one wavelength per path (the reference's default,
     * `hwss false`: IntegrateRayNM), lambda_min + floor(u * num_wavelengths) *
     * (lambda_max - lambda_min) / num_wavelengths when 0 < num_wavelengths <
     * 10000, else uniform in the range.  spectral_samples (0 = 1) paths are
     * traced per pixel sample and averaged (nSpectralSamples); each draws its
     * own position in the pixel.  Adaptive sampling needs spectral_samples 1. */
    int32_t spectral_mode;
    int32_t num_wavelengths;
    int32_t spectral_samples;
} rtb200_render_settings;

#define RTB200_SPECTRAL_HWSS 0
#define RTB200_SPECTRAL_SINGLE 1

/* Random numbers of the path decisions.  HASH: a counter-based hash of
 * (seed, pixel, sample, dimension) with a fixed dimension layout.  SOBOL: the
 * reference's sampler (Utilities/SobolSampler.h, Sampling/SobolSequence.h:55-206):
 * Owen-scrambled padded Sobol (dimension d uses Sobol dimension d & 1 scrambled
 * with HashCombine(seed, d)), the pixel's seed HashCombine(x, y) (rows from the
 * top; with a nonzero job seed s, HashCombine(HashCombine(x, y), s)), sample
 * index = the pixel's sample number; bounce `depth` draws dimensions
 * (16 + depth) * 32 + j in the order the reference's integrator consumes them
 * (StartStream(16 + depth), PathTracingIntegrator.cpp:4112), camera jitter and
 * the hero wavelength dimensions 0, 1, 2.  With one seed per pixel, and
 * dimension pairs that replay one Sobol pair under another scramble, a pixel
 * rendered this way does not converge to its integral (the reference's
 * images carry the same per-pixel error).  SOBOL_SHUFFLED: the same with the
 * sample index first Owen-scrambled by a seed per dimension pair (Burley's
 * decorrelation of padded dimensions, JCGT 9(4), 2020), which keeps the
 * stratification and converges. */
#define RTB200_SAMPLER_HASH 0
#define RTB200_SAMPLER_SOBOL 1
#define RTB200_SAMPLER_SOBOL_SHUFFLED 2

/* Next-event luminary selection.  BVH: the reference's light BVH
 * (Lights/LightBVH.cpp: importance = power / squared distance to the node's
 * box, one random number rescaled down the tree; its pdf enters the MIS
 * weights) when the scene has more than one luminary, as the reference does
 * by default (StabilityConfig::useLightBVH, LightSampler.cpp:748-761).
 * POWER: in proportion to emitted power alone (the reference's alias table,
 * light_bvh false). */
#define RTB200_LIGHTS_BVH 0
#define RTB200_LIGHTS_POWER 1

/* Pixel filters.  BOX: uniform jitter in the pixel, the pixel is the mean of
 * its own samples.  GAUSSIAN: the reference's GaussianPixelFilter
 * (Sampling/GaussianPixelFilter.h:40-127).  With a half-width above 0.501
 * pixel every sample is splatted into the pixels within the support and a
 * pixel resolves to sum(w XYZ) / sum(w), 0 where sum(w) <= 1e-10
 * (PixelBasedRasterizerHelper.cpp:143-149, FilteredFilm.cpp:42-132); a
 * narrower kernel instead moves each camera sample by the truncated
 * Gaussian about the pixel centre and averages the pixel's own samples
 * (PathTracingSpectralRasterizer.cpp:321-331). */
#define RTB200_FILTER_BOX 0
#define RTB200_FILTER_GAUSSIAN 1

typedef struct rtb200_job rtb200_job;

typedef struct {
    int64_t spp;              /* samples per pixel rendered so far */
    int64_t samples;          /* camera samples (paths) */
    int64_t segments;         /* extended rays */
    int64_t shadow_rays;
    double seconds;           /* device time of all render calls */
    int64_t active_pixels;    /* pixels still sampled (adaptive: not yet converged nor at the maximum) */
} rtb200_stats;

/* A job holds the path pool, queues and film of one image on the device.
 * rtb200_job_render adds spp samples per pixel and returns when they are in
 * the film (PixelBasedRasterizerHelper::RasterizeScene's progressive passes,
 * Rendering/PixelBasedRasterizerHelper.cpp:982-1440, with the per-pixel loop
 * of PathTracingSpectralRasterizer::IntegratePixel,
 * Rendering/PathTracingSpectralRasterizer.cpp:206-479).
 * rtb200_job_read_film writes width*height*3 floats: the mean XYZ per pixel
 * over all samples so far (rows top to bottom); RTB200_E_NOT_READY while a
 * request of the job is in flight on an engine.
 *
 * Adaptive sampling (adaptive_max_spp > 0; AdaptiveSamplingConfig,
 * Utilities/AdaptiveSamplingConfig.h, and the per-pixel loop of
 * PathTracingSpectralRasterizer.cpp:256-410): each render call is one batch
 * of spp samples for every pixel that has not converged, capped at
 * adaptive_max_spp samples per pixel.  After the batch, a pixel with at least
 * 32 samples converges when the standard error of its luminance (XYZ.Y) over
 * its mean is below adaptive_threshold * (1 - 4 / N), or, for a black pixel,
 * when the sum of squared deviations is below 1e-12 after 64 samples.  A
 * pixel's value is the mean of its own samples (box filter) or the splat of
 * all samples taken (Gaussian).  rtb200_stats.active_pixels says how many
 * pixels the next call samples; a call with none left returns RTB200_OK and
 * renders nothing.  rtb200_job_read_sample_counts writes the samples each
 * pixel took (width*height uint32; the reference's sample map is counts /
 * adaptive_max_spp). */
int rtb200_job_create(rtb200_scene* scene, const rtb200_render_settings* settings, rtb200_job** out);
int rtb200_job_render(rtb200_job* job, int32_t spp);
int rtb200_job_read_film(rtb200_job* job, float* xyz);
int rtb200_job_read_sample_counts(rtb200_job* job, uint32_t* counts);

/* Film to colour.  rtb200_job_read_rgb writes width*height*3 floats: each
 * pixel's XYZ (as rtb200_job_read_film returns it) converted to linear
 * Rec.709 RGB the way the rasterizer resolves a pixel, RISEPel(XYZPel)
 * (ColorUtils::XYZtoRec709RGB, Utilities/Color/Color.cpp:214-228, with its
 * chromaticity gamut move, Utilities/Color/ColorUtils.cpp:232-363).
 * rtb200_job_read_display writes width*height*3 bytes for an 8-bit image
 * file: that RGB scaled by 2^exposure_ev, passed through the tone curve
 * (DisplayTransformWriter::WriteColor, Rendering/DisplayTransformWriter.cpp:45-62;
 * curves of Rendering/DisplayTransform.h:80-222), sRGB-encoded, clamped to
 * [0, 1] and truncated to 0..255 (the PNG / PPM / TGA writers'
 * Integerize<sRGBPel>, e.g. RasterImages/PPMWriter.cpp WriteColor). */
#define RTB200_TONE_NONE 0      /* clip negatives and non-finite values to 0 */
#define RTB200_TONE_REINHARD 1
#define RTB200_TONE_ACES 2
#define RTB200_TONE_AGX 3
#define RTB200_TONE_HABLE 4
int rtb200_job_read_rgb(rtb200_job* job, float* rgb);
int rtb200_job_read_display(rtb200_job* job, float exposure_ev, int32_t tone, uint8_t* rgb8);
int rtb200_job_stats(const rtb200_job* job, rtb200_stats* out);

/* Progress of a render (IRasterizer::SetProgressCallback with
 * IProgressCallback::Progress, Interfaces/IProgressCallback.h:20-50; called
 * by PixelBasedRasterizerHelper between regions, which stops the render when
 * it returns false, PixelBasedRasterizerHelper.cpp:1512-1530).  While
 * rtb200_job_render or rtb200_engine_render runs, fn(user, progress, total)
 * is called on the calling thread after every engine step with the pixel
 * samples finished so far and asked for in this call (progress is
 * fractional: paths finished / paths per pixel sample).  Returning 0 stops
 * the request: no new pixel samples start, those already started finish,
 * every pixel keeps the same whole number of samples, and the call returns
 * RTB200_E_CANCELLED with the film holding them.  fn runs with the
 * context's lock held and must not call into rtb200 on the same context.
 * fn = null removes the callback. */
typedef int32_t (*rtb200_progress_fn)(void* user, double progress, double total);
int rtb200_job_set_progress(rtb200_job* job, rtb200_progress_fn fn, void* user);
/* relMSE of the job's film against a reference image (width*height*3 host
 * floats, XYZ): the mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2),
 * reduced on the device in FP64.  Films keep a Kahan-compensated FP32 running
 * sum up to 4096 samples per pixel and an FP64 one beyond.  No counterpart in
 * the reference (its convergence tests compare images on the host). */
int rtb200_job_relmse(rtb200_job* job, const float* ref_xyz, double* relmse);
int rtb200_job_destroy(rtb200_job* job);

/* ---- engines: many jobs in one wavefront -------------------------------- */

/* An engine owns a device pool of `capacity` path slots (0 = 2^21), the
 * ray and shadow-ray queues, and a table of up to 1024 jobs.  Jobs of
 * different scenes and resolutions (same BVH layout) share its wavefront:
 * every iteration hands free path slots to whichever jobs still have samples
 * to give, so their work overlaps on the device.  No counterpart in the
 * reference, which renders one image at a time
 * (PixelBasedRasterizerHelper::RasterizeScene,
 * Rendering/PixelBasedRasterizerHelper.cpp:982-1440).
 *
 * rtb200_engine_render: render spp[i] more samples per pixel for each
 *   jobs[i] in one shared wavefront and return when all are in the films;
 *   use_graph replays the iterations from a captured CUDA graph.
 * Continuous batching: rtb200_engine_submit adds a job with a request of
 *   spp samples per pixel (allowed while other jobs are in flight);
 *   rtb200_engine_step runs `iterations` wavefront iterations over all
 *   submitted jobs; rtb200_engine_progress reports samples finished / total
 *   of a job's request as of the last step; rtb200_engine_retire folds a
 *   finished request into the job's film (RTB200_E_NOT_READY before that)
 *   and removes the job from the engine. */
typedef struct rtb200_engine rtb200_engine;
int rtb200_engine_create(rtb200_ctx* ctx, int32_t capacity, rtb200_engine** out);
int rtb200_engine_render(rtb200_engine* engine, rtb200_job* const* jobs, const int32_t* spp, int32_t n,
                         int32_t use_graph);
int rtb200_engine_submit(rtb200_engine* engine, rtb200_job* job, int32_t spp);
int rtb200_engine_step(rtb200_engine* engine, int32_t iterations, int32_t use_graph);
int rtb200_engine_progress(const rtb200_engine* engine, const rtb200_job* job, int64_t* done, int64_t* total);
int rtb200_engine_retire(rtb200_engine* engine, rtb200_job* job);
/* Stops a submitted job's request as a progress callback returning 0 does:
 * no new pixel samples start; after the samples started finish, progress
 * reports done == total and the job can be retired (a served request that
 * is abandoned or cancelled by its client). */
int rtb200_engine_cancel(rtb200_engine* engine, rtb200_job* job);
int rtb200_engine_destroy(rtb200_engine* engine);
/* Wavefront iterations rtb200_engine_render runs between host polls of the
 * jobs' progress (default 4; rounded up to even, 2 .. 1024).  Fewer polls
 * save host round trips, more let a finished batch stop sooner; the project's
 * autotuner (rise_b200/autotune.py) picks it with the pool capacity. */
int rtb200_engine_set_poll(rtb200_engine* engine, int32_t iterations);

/* ---- host BVH build and export ----------------------------------------- */

/* Builds the reference BVH on the host (all cores) without a device and
 * exposes its node arrays: BVH2 nodes in the reference's 32-byte packing,
 * the leaf-order triangle indices, and the collapsed 128-byte BVH4 nodes.
 * Replaces BVH::Serialize's node/index export
 * (Acceleration/BVH.h:353-373) and the BVH4 collapse (BVH.h:477-642). */
typedef struct rtb200_bvh_host rtb200_bvh_host;
int rtb200_bvh_host_build(const float* tri9, int64_t n_tri, int32_t threads, rtb200_bvh_host** out);
int rtb200_bvh_host_info(const rtb200_bvh_host* h, int64_t* n_nodes2, int64_t* n_nodes4);
/* Any output pointer may be NULL.  nodes2: 32 * n_nodes2 bytes;
 * prims: n_tri uint32; nodes4: 128 * n_nodes4 bytes. */
int rtb200_bvh_host_export(const rtb200_bvh_host* h, void* nodes2, uint32_t* prims, void* nodes4);
int rtb200_bvh_host_destroy(rtb200_bvh_host* h);
/* The same for a .risemesh: its cached BVH2 as the scene commit would adopt
 * it (checked, then collapsed), or the reference build of its triangles when
 * the file has no cache or use_cached_bvh is 0. */
int rtb200_bvh_host_from_risemesh(const rtb200_risemesh* mesh, int32_t use_cached_bvh, rtb200_bvh_host** out);

/* ---- batched ray casting ----------------------------------------------- */

/* Host buffers: copies rays to the device, casts, copies results back, and
 * returns when the results are in `hits` / `occluded`. */
int rtb200_cast_closest(rtb200_scene* scene, const rtb200_ray* rays, int64_t n, rtb200_hit* hits);
int rtb200_cast_any(rtb200_scene* scene, const rtb200_ray* rays, int64_t n, uint8_t* occluded);

/* Device buffers (device pointers), asynchronous on `stream`, a
 * cudaStream_t taken as is (NULL is the CUDA default stream, as everywhere
 * in CUDA).  The caller synchronises.  Every cast on one scene uses the
 * scene's one work counter (the atomic that hands rays to warps): casts on
 * the same scene whose work overlaps on the GPU (different streams or host
 * threads) race on it and must be ordered by the caller, e.g. on one stream.
 * The kernels record a traversal-stack overflow in the scene's device error
 * word instead of failing; commit refuses BVHs whose exact stack bound the
 * kernels cannot hold, so it stays clear for committed scenes, and
 * rtb200_scene_device_status reads it: it waits for `stream`, returns
 * RTB200_E_DEVICE (and clears the word) if any cast on the scene since the
 * last check set it, else RTB200_OK. */
int rtb200_cast_closest_device(rtb200_scene* scene, const rtb200_ray* d_rays, int64_t n,
                               rtb200_hit* d_hits, void* stream);
int rtb200_cast_any_device(rtb200_scene* scene, const rtb200_ray* d_rays, int64_t n,
                           uint8_t* d_occluded, void* stream);
int rtb200_scene_device_status(rtb200_scene* scene, void* stream);

/* Closest hit that allocates no device memory (no counterpart in the
 * reference: the reference renderer allocates on the host and never on a
 * GPU).  For callers that must not call cudaMalloc/cudaFree when they cast
 * rays -- e.g. a host application whose pool allocator owns all device
 * memory, or a latency-critical thread that cannot afford the device-wide
 * synchronisation cudaMalloc/cudaFree may cause.  Same kernel and results as
 * rtb200_cast_closest_device; the kernel's scratch (work counter, error
 * word) lives in a static RTB200_NOALLOC_SCRATCH_BYTES-byte device array,
 * one per GPU, held until the process exits.  The first call on a device
 * looks up that array's address (no allocation); make that first call
 * before any stream capture.  Every call shares the array and clears it on
 * its stream first, so calls whose work overlaps on the GPU race on it and
 * must be serialised by the caller.  At most RTB200_NOALLOC_MAX_RAYS rays per
 * call; larger n is rejected with RTB200_E_INVALID.  The kernel's error word
 * (a traversal-stack overflow, which commit's exact stack bound rules out for
 * committed scenes) sits in the same array and is not reported by this entry:
 * reading it would need a synchronisation this entry exists to avoid. */
#define RTB200_NOALLOC_SCRATCH_BYTES 256
#define RTB200_NOALLOC_MAX_RAYS 2147483647LL
int rtb200_cast_closest_noalloc(rtb200_scene* scene, const rtb200_ray* d_rays, int64_t n,
                                rtb200_hit* d_hits, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RTB200_H */
