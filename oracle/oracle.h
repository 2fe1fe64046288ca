/* oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement ("port") of the reference renderer's hot-path algorithms:
 * the SAH-binned BVH builder, its BVH4 collapse and traversal, the
 * double-precision Moller-Trumbore ray/triangle test, and (pt_oracle.cpp) the
 * hero-wavelength spectral path tracer.  Every function cites the reference
 * file:line it follows.  Only tests/, the smoke check and bench.py's CPU
 * baseline leg load this library; the product never does.
 */
#ifndef RTB200_ORACLE_H
#define RTB200_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same 32-byte packing as the reference BVH2 node
 * (src/Library/Acceleration/BVH.h:87-96). */
typedef struct {
    float    bmin[3];
    float    bmax[3];
    uint32_t first_or_left;
    uint16_t count;
    uint8_t  axis;
    uint8_t  pad;
} orc_node2;

/* Same 128-byte packing as the reference BVH4 node (BVH.h:124-137). */
typedef struct {
    float    minx[4], miny[4], minz[4];
    float    maxx[4], maxy[4], maxz[4];
    int32_t  child[4];
    uint16_t count[4];
    uint8_t  nchild;
    uint8_t  axis;
    uint8_t  pad[6];   /* the reference node is alignas(16): 128 bytes */
} orc_node4;

typedef struct orc_bvh orc_bvh;

orc_bvh* orc_bvh_build(const float* tri9, int64_t n_tri);
void     orc_bvh_destroy(orc_bvh* b);
int64_t  orc_bvh_num_nodes2(const orc_bvh* b);
int64_t  orc_bvh_num_nodes4(const orc_bvh* b);
void     orc_bvh_export(const orc_bvh* b, orc_node2* nodes2, uint32_t* prims, orc_node4* nodes4);

/* rays: 8 floats each (ox,oy,oz,tmin, dx,dy,dz,tmax). */
void orc_closest(const orc_bvh* b, const float* rays, int64_t n, int32_t* id, double* t,
                 double* edge_dist, int threads);
void orc_any(const orc_bvh* b, const float* rays, int64_t n, uint8_t* occ, int threads);
/* Brute force over every triangle (small cases only). */
void orc_closest_brute(const float* tri9, int64_t n_tri, const float* rays, int64_t n,
                       int32_t* id, double* t);
int  orc_ray_triangle(const double* o, const double* d, const double* v0, const double* ea,
                      const double* eb, double* t, double* alpha, double* beta);

/* Spectral path tracer (pt_oracle.cpp): renders the mean XYZ of `spp`
 * samples per pixel (samples sample_begin .. sample_begin + spp - 1) over the
 * crop [x0, x1) x [y0, y1) into xyz (3 doubles per crop pixel, row-major).
 *   meshes: n_mesh x 4 int64 (first triangle, count, material, double sided)
 *   spectra: the spectrum table of n_spec ids: a header of 4 floats per id,
 *           {0, 380, 780, offset} for 81 samples on the 5 nm grid or
 *           {n, begin, end, offset} for a binned packet, {-1, 380, 780, offset}
 *           for an RGB colour's sigmoid (c0, c1, c2, scale), {-2, 0, 1e30, offset}
 *           for a black body (temperature, scale), then the samples
 *   mats_i: n_mat x 5 int32 (type, reflectance, emission, eta, kappa)
 *   mats_f: n_mat x 2 float (alpha, ior)
 *   cam:    10 doubles (pos, look, up, vertical fov in degrees)
 *   setd:   6 doubles (lambda_min, lambda_max, rr_threshold, filter size, filter sigma,
 *           adaptive threshold)
 *   points: n_point x 7 doubles (position, colour, power) of point lights
 *   nrm9:   n_tri x 9 floats, the vertex normals of each triangle's corners
 *           (all zero: a flat triangle), or null
 *   seti:   17 int32 (width, height, max_depth, rr_min_depth, nee_per_lambda, seed, filter,
 *           adaptive maximum samples per pixel or 0, light selection: 0 light BVH, 1 power,
 *           sampler: 0 hash, 1 Owen-scrambled Sobol, 2 the same with shuffled indices,
 *           bounce limits on, maximum diffuse, glossy and transmission bounces,
 *           spectral mode: 0 hero + 3 companions, 1 one wavelength per path,
 *           wavelength bins of the single mode (0 = continuous), spectral samples
 *           per pixel sample)
 * A dielectric whose eta (mats_i column 3) names a spectrum refracts with that
 * index per wavelength; where the hero's and a companion's differ, the
 * companions end and the hero continues alone.
 * filter 0 is the box film (mean of the pixel's own samples); filter 1 is the
 * Gaussian pixel filter: with size / 2 > 0.501 the samples of every pixel
 * within the support are splatted and a pixel is sum(w XYZ) / sum(w); a
 * narrower kernel warps each camera sample about the pixel centre instead.
 * Adaptive sampling (seti[7] = maximum samples per pixel > 0, setd[5] = its
 * threshold): every pixel takes batches of `spp` samples from sample 0 until
 * its luminance estimate converges or the maximum is reached (sample_begin
 * must be 0); a pixel is the mean of its own samples (box, warped) or the
 * splat of every sample taken (Gaussian).  counts (nullable) receives the
 * samples each crop pixel took.
 *   envi:   2 int32 (environment spectrum or -1, visible)
 *   cie:    3 x 81 doubles, the reference's CIE 1931 table (x, y, z bars)
 *   env_image: an image environment (replaces the uniform sky) or null
 * Returns 0 on success. */
typedef struct {
    const float* rgb;        /* width x height x 3 linear Rec.709, rows top to bottom */
    int32_t width, height;
    double scale;            /* radiance_scale */
    double orient_rad[3];    /* radiance_orient, radians */
    const float* uplift;     /* the Jakob-Hanika table, 3 x 64^3 x 3 floats */
} OrcEnvImage;
int orc_pt_render(const float* tri9, int64_t n_tri, const int64_t* meshes, int32_t n_mesh,
                  const float* spectra, int32_t n_spec, const int32_t* mats_i, const float* mats_f,
                  int32_t n_mat, const int32_t* envi, const double* cam, const double* setd,
                  const int32_t* seti, int32_t spp, int32_t sample_begin, int32_t x0, int32_t y0,
                  int32_t x1, int32_t y1, int32_t threads, double* xyz, const double* cie,
                  int32_t* counts, int32_t n_point, const double* points,
                  const float* nrm9, const OrcEnvImage* env_image);

/* Building blocks of the path-tracing oracle, exported so tests can hold each
 * against the reference's own code (oracle/_ref/libref_pt.so). */
double orc_pt_gaussian_weight(double size, double sigma, double dx, double dy);
void   orc_pt_light_bvh(int n, const double* pos, const double* power, int m, const double* pts, const double* xi,
                        int* picked, double* pdf, double* pdf_all);
void   orc_pt_xyz_to_rec709(const double* xyz, double* rgb);
void   orc_pt_display(const double* rgb, double exposure_ev, int tone, unsigned char* out3);
void   orc_pt_sample_wavelengths(double u, double lmin, double lmax, double* lam4);
int    orc_pt_xyz_from_nm(double nm, const double* cie, double* xyz3);
double orc_pt_ggx_d(double alpha, double cos_h);
double orc_pt_ggx_lambda(double alpha, double cos_t);
double orc_pt_ggx_g2(double alpha, double cos_i, double cos_o);
void   orc_pt_vndf_sample(const double* wi, const double* t, const double* b, const double* n, double alpha,
                          double u1, double u2, double* m);
double orc_pt_vndf_pdf(const double* wi, const double* wo, const double* n, double alpha);
double orc_pt_conductor_f(double cos_i, double ni, double nt, double k);
double orc_pt_dielectric_r(double cos_i, double cos_t, double ni, double nt);
double orc_pt_lookup_ess(double c, double alpha);
double orc_pt_lookup_eavg(double alpha);
double orc_pt_ms_z(double alpha);
double orc_pt_ms_pdf(double c, double alpha, double z);
double orc_pt_ms_sample_cos(double alpha, double u);
double orc_pt_fresnel_avg(double ni, double nt, double k);
double orc_pt_fms(double favg, double eavg);
double orc_pt_power_heuristic(double a, double b);
int    orc_pt_russian_roulette(int depth, int min_depth, double threshold, double cur, double prev, double u,
                               double* survival);
/* The reference's padded Owen-scrambled Sobol (Sampling/SobolSequence.h):
 * the 32-bit scrambled value per (index, dimension, seed), and HashCombine. */
void   orc_pt_sobol(const uint32_t* index, const uint32_t* dim, const uint32_t* seed, int64_t n, uint32_t* out);
void   orc_pt_hash_combine(const uint32_t* a, const uint32_t* b, int64_t n, uint32_t* out);
void   orc_pt_tables(double* ess, double* eavg);
void   orc_pt_set_tables(const double* ess, const double* eavg);

#ifdef __cplusplus
}
/* Double-precision ray queries used by the path-tracing oracle. */
int32_t orc_closest_d(const orc_bvh* h, const double o[3], const double d[3], double* t);
bool orc_any_d(const orc_bvh* h, const double o[3], const double d[3], double tmax);
#endif
#endif
