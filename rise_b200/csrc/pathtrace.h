// pathtrace.h -- host interface to the wavefront path-tracer kernels.
#pragma once
#include <cuda_runtime.h>

#include "pt_types.h"

namespace rtb200 {

// Everything one wavefront iteration needs.  `jobs` is the device job table;
// `ids` (device) lists the table entries that may receive new samples, and
// queues.cnt[kCntJobs] (device) how many there are, so a captured iteration
// serves any number of jobs.  Every job in one engine uses the same BVH layout.
struct PtLaunch {
    const PtJobDev* jobs;
    const int* ids;
    int layout;
    bool spill;        // some job's BVH needs the local-memory stack continuation
    bool uniform;      // every job renders `scene`
    bool classify;     // some job's scene mixes shading classes: sort paths before shading
    int shade_class;   // without sorting: the one shading class of every job's scene, or -1
    bool env_image;    // some job's scene has an image environment (shading kernels carry its code)
    PtScene scene;
    PtPaths paths;
    PtQueues queues;
    int sms;
};

// One wavefront iteration (regenerate, extend, shade, connect, swap counters),
// asynchronous on `st`.  The caller swaps queues.active/active_next and
// queues.free_/free_next after each call.
cudaError_t PtIteration(const PtLaunch& L, int iter, cudaStream_t st);
// Splat paths still marked finished into their films (end of a render).
cudaError_t PtDrain(const PtLaunch& L, cudaStream_t st);
// Upload the GGX E_ss (32 x 32), E_avg (32), multiple-scattering lobe
// normalisation (32) and cumulative segment integral (32 x 34) tables.
cudaError_t PtSetGgxTables(const float* ess, const float* eavg, const float* msz, const float* mscum,
                           const float* favg_x, const float* favg_w);
// Fold a film of this request (n floats) into the compensated running sums
// and clear it.
cudaError_t PtFold(float* pass, float* sum, float* comp, int n, int sms, cudaStream_t st);
// The same into an FP64 running sum (first: move the FP32 sums over first).
cudaError_t PtFoldWide(float* pass, float* sum, float* comp, double* wide, int n, bool first, int sms,
                       cudaStream_t st);
// *out = sum over pixels and XYZ channels of (x - r)^2 / (r^2 + 1e-2), x the
// resolved film (channels 3: sum * inv_spp, or sum / counts[pixel] when
// counts is given; 4: weighted sum / weight), r the device reference; FP64
// accumulation.
cudaError_t PtRelMse(const float* sum, const float* comp, const double* wide, const unsigned* counts,
                     const float* ref, int npix, int channels, double inv_spp, double* out, int sms, cudaStream_t st);
// Resolve the film to colour (resolve.cu): linear Rec.709 into rgb (3 floats
// per pixel) when rgb is given, else 8-bit sRGB after exposure (ev_mul) and
// the RTB200_TONE_* curve into rgb8.
cudaError_t PtResolveColor(const float* sum, const float* comp, const double* wide, const unsigned* counts,
                           int channels, double inv_spp, int npix, double ev_mul, int tone, float* rgb,
                           unsigned char* rgb8, int sms, cudaStream_t st);
// Adaptive sampling after a batch: count[p] += batch for the n listed pixels,
// convergence test, and the pixels left to sample appended to next (*n_next,
// zeroed first).
cudaError_t PtConverge(const unsigned* list, int n, const double* lum, unsigned* count, int batch, int max_spp,
                       double threshold, unsigned* next, int* n_next, int sms, cudaStream_t st);

}  // namespace rtb200
