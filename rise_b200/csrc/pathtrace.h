// pathtrace.h -- host interface to the wavefront path-tracer kernels.
#pragma once
#include <cuda_runtime.h>

#include "pt_types.h"

namespace rtb200 {

struct PtLaunch {
    PtScene scene;
    PtPaths paths;
    PtQueues queues;
    PtFilm film;
    PtJobParams params;
    int sms;
};

// One wavefront iteration (regenerate, extend, shade, connect, swap counters),
// asynchronous on `st`.  The caller swaps queues.active/active_next and
// queues.free_/free_next after each call.
cudaError_t PtIteration(const PtLaunch& L, cudaStream_t st);
// Upload the GGX E_ss (32 x 32) and E_avg (32) tables to constant memory.
cudaError_t PtSetGgxTables(const float* ess, const float* eavg);
// Fold this call's film into the compensated running sums and clear it.
cudaError_t PtFold(const PtFilm& F, int npix, int sms, cudaStream_t st);

}  // namespace rtb200
