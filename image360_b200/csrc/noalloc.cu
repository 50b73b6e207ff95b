// Allocation-free variant of the device seam blend (i360b_launch_blend).
//
// Some callers must not allocate device memory once they are running: hosts
// that reserve the GPU's memory up front for their own pool (a cudaMalloc then
// fails or breaks their budget), and latency-critical render loops in which a
// cudaMalloc/cudaFree would synchronise the whole device.  For them this entry
// point takes every byte of scratch the blend needs (coverage bits, chamfer
// fields, owner map, pyramid levels, seam state and its own work tables) from
// one static device array compiled into the library, and allocates nothing.
//
// The array is a fixed kNoAllocScratchBytes per device; every GPU that loads
// the library holds it until the process exits.  A chunk whose scratch would
// exceed it is rejected with I360B_INVALID_PARAM before anything is enqueued.
// All calls share the array and each call overwrites what the previous one
// left there, so calls whose GPU work overlaps (two threads, or two streams)
// race; serialise them.  i360b_initialize looks up the array's device
// address on the device it selects (with that device current), which makes
// the runtime load this file's module - and so reserve the 12 MiB - at
// initialisation, not on the first call; a call on a device that was not set
// up that way looks it up then.
#include "common.cuh"

#include <mutex>

namespace i360b
{
namespace
{
// 12 MiB: a 256x256 chunk with 8 contributors needs about 8.5 MiB.
constexpr size_t kNoAllocScratchBytes = size_t(12) << 20;

__device__ __align__(256) unsigned char g_noallocScratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noallocMu;
void* g_noallocPtr[kMaxDevices] = {};

}  // namespace

// Device address of the scratch array on the current device (host code only
// sees a stand-in for the symbol, never its device address).
int noalloc_scratch(void** out)
{
    int dev = -1;
    I360B_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(I360B_CUDA_ERROR, "Device index %d out of range.", dev);
    std::lock_guard<std::mutex> lk(g_noallocMu);
    if (!g_noallocPtr[dev])
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess || !p) return cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "cudaGetSymbolAddress");
        g_noallocPtr[dev] = p;
    }
    *out = g_noallocPtr[dev];
    return I360B_SUCCESS;
}
}  // namespace i360b

using namespace i360b;

extern "C" int i360b_launch_blend_noalloc(const unsigned short* const* dWarped, int numContributors, int width,
                                          int height, int numBands, unsigned short* dOut, void* stream)
{
    clear_error();
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    if (!dOut || (numContributors > 0 && !dWarped)) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    if (numContributors < 0 || numContributors > 127) return fail(I360B_INVALID_PARAM, "numContributors must be 0-127.");
    if (numBands < 1) return fail(I360B_INVALID_PARAM, "numBands must be >= 1.");
    for (int i = 0; i < numContributors; ++i)
        if (!dWarped[i]) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    void* scratch = nullptr;
    I360B_TRY(noalloc_scratch(&scratch));
    return launch_blend_chunk_in(scratch, kNoAllocScratchBytes, dWarped, numContributors, width, height, numBands, dOut,
                                 static_cast<cudaStream_t>(stream));
}
