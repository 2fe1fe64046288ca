// noalloc.cu -- closest-hit casting that allocates no device memory.
//
// Some callers cannot allocate device memory at the time they cast rays: a
// host application that hands the whole GPU to its own pool allocator and
// forbids further cudaMalloc calls, or a caller on a latency-critical thread
// that must not run cudaMalloc/cudaFree because they can synchronise the
// whole device.  rtb200_cast_closest_noalloc serves them: it runs the same
// closest-hit kernel as rtb200_cast_closest_device, but the kernel's scratch
// (the work counter that hands rays to warps, and the error word) lives in
// the file-scope device array below instead of in memory the scene owns.
//
// The array is RTB200_NOALLOC_SCRATCH_BYTES (256) bytes and exists once per
// GPU that loads the library, until the process exits.  Every call shares it
// and it keeps the last call's contents, so each call clears the counter and
// the error word on its stream before launching; two calls whose work
// overlaps on the GPU (different streams, or different host threads) race on
// it and must be serialised by the caller.
#include <mutex>
#include <string>

#include "core.h"

namespace {

constexpr size_t kScratchBytes = RTB200_NOALLOC_SCRATCH_BYTES;
constexpr size_t kCounterOffset = 0;   // unsigned long long work counter
constexpr size_t kErrorOffset = 64;    // unsigned error word (own cache sector)
static_assert(kErrorOffset + sizeof(unsigned) <= kScratchBytes, "scratch layout exceeds the array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per CUDA device, looked up once.  In
// host code the array's name is a host-side stand-in, not a device address,
// so the kernel must be given the address cudaGetSymbolAddress returns.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

cudaError_t ScratchAddress(int device, void** out)
{
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[device] = p;
    }
    *out = g_addr[device];
    return cudaSuccess;
}

}  // namespace

using namespace rtb200;

extern "C" int rtb200_cast_closest_noalloc(rtb200_scene* s, const rtb200_ray* d_rays, int64_t n,
                                           rtb200_hit* d_hits, void* stream)
{
    if (!s) return RTB200_E_INVALID;
    rtb200_ctx* ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!s->committed) return SetError(ctx, RTB200_E_INVALID, "scene not committed");
    if (n < 0 || (n > 0 && (!d_rays || !d_hits))) return SetError(ctx, RTB200_E_INVALID, "bad ray buffers");
    if (n > (int64_t)RTB200_NOALLOC_MAX_RAYS)
        return SetError(ctx, RTB200_E_INVALID,
                        "rtb200_cast_closest_noalloc: " + std::to_string(n) + " rays exceed the limit of " +
                            std::to_string((long long)RTB200_NOALLOC_MAX_RAYS) + " rays per call");
    if ((((uintptr_t)d_rays) & 15u) || (((uintptr_t)d_hits) & 15u))
        return SetError(ctx, RTB200_E_INVALID, "ray/hit buffers must be 16-byte aligned");
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return SetError(ctx, RTB200_E_INVALID, "device index out of range");
    if (n == 0) return RTB200_OK;
    cudaError_t e = cudaSetDevice(ctx->device);
    void* base = nullptr;
    if (e == cudaSuccess) e = ScratchAddress(ctx->device, &base);
    if (e != cudaSuccess) return CudaCheck(ctx, e, "scratch symbol lookup");
    const cudaStream_t st = (cudaStream_t)stream;
    // The array keeps the previous call's counter: clear it (and the error
    // word) on this call's stream before the kernel reads it.
    e = cudaMemsetAsync(base, 0, kScratchBytes, st);
    if (e == cudaSuccess)
        e = LaunchCastClosestScratch(s, d_rays, n, d_hits,
                                     (unsigned long long*)((char*)base + kCounterOffset),
                                     (unsigned*)((char*)base + kErrorOffset), st);
    return CudaCheck(ctx, e, "closest-hit launch (no-alloc)");
}
