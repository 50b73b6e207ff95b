// Runtime plumbing: device selection, per-thread error strings and streams,
// and the stream-ordered device memory pool.
//
// The reference backend allocates and frees device memory on every call
// (CudaPipeline.cpp:207-267); here every allocation comes from the device's
// CUDA memory pool with its release threshold raised to "never", so after the
// first call of a given size the pool serves it without touching the driver.
#include "common.cuh"

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace i360b
{
namespace
{
std::mutex g_mu;
std::atomic<bool> g_init{false};
int g_device = -1;
int g_sms = 0;
std::atomic<unsigned> g_generation{0};  // bumped by shutdown so thread streams are recreated

thread_local char t_err[512] = {0};
thread_local cudaStream_t t_stream = nullptr;
thread_local unsigned t_stream_gen = ~0u;
}  // namespace

int fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(t_err, sizeof(t_err), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { t_err[0] = 0; }

int cuda_fail(cudaError_t e, const char* what)
{
    int code = I360B_CUDA_ERROR;
    if (e == cudaErrorMemoryAllocation) code = I360B_OUT_OF_MEMORY;
    else if (e == cudaErrorLaunchFailure || e == cudaErrorLaunchOutOfResources || e == cudaErrorInvalidConfiguration ||
             e == cudaErrorNoKernelImageForDevice)
        code = I360B_KERNEL_LAUNCH_FAILED;
    else if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        code = I360B_NO_GPU;
    return fail(code, "%s: %s", what, cudaGetErrorString(e));
}

namespace
{
// Armed host-side failures (i360b_debug_inject_failure).
std::atomic<int> g_injectAlloc{0}, g_injectLaunch{0};

bool take_injected(std::atomic<int>& n)
{
    int v = n.load();
    while (v > 0)
        if (n.compare_exchange_weak(v, v - 1)) return true;
    return false;
}
}  // namespace

bool inject_alloc_failure() { return take_injected(g_injectAlloc); }

int check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what);
    if (take_injected(g_injectLaunch)) return fail(I360B_KERNEL_LAUNCH_FAILED, "%s: launch failed (injected)", what);
    return I360B_SUCCESS;
}

bool initialized() { return g_init.load(); }
int device() { return g_device; }
int sm_count() { return g_sms; }

static int do_initialize()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0)
    {
        cudaGetLastError();
        return fail(I360B_NO_GPU, "No CUDA device found (%s).", e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
    }
    // Same selection rule as CudaPipeline::Initialize: the device with the
    // most memory; only compute capability 10.x (sm_100a code) qualifies.
    int best = -1;
    size_t bestMem = 0;
    for (int d = 0; d < n; ++d)
    {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, d) != cudaSuccess) continue;
        if (p.major != 10) continue;
        if (best < 0 || p.totalGlobalMem > bestMem)
        {
            best = d;
            bestMem = p.totalGlobalMem;
        }
    }
    if (best < 0) return fail(I360B_NO_GPU, "No compute-capability 10.x (B200-class) device among %d device(s).", n);
    I360B_CUDA(cudaSetDevice(best), "cudaSetDevice");
    cudaMemPool_t pool;
    I360B_CUDA(cudaDeviceGetDefaultMemPool(&pool, best), "cudaDeviceGetDefaultMemPool");
    uint64_t threshold = ~0ull;
    I360B_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "cudaMemPoolSetAttribute");
    I360B_CUDA(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, best), "cudaDeviceGetAttribute");
    g_device = best;
    // Resolve the allocation-free blend's scratch array now, with the device
    // current: this loads its module, so the array is reserved here rather
    // than inside that entry point's first call.
    void* scratch = nullptr;
    I360B_TRY(noalloc_scratch(&scratch));
    g_init.store(true);
    return I360B_SUCCESS;
}

int ensure_ready()
{
    if (g_init.load())
    {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != g_device) I360B_CUDA(cudaSetDevice(g_device), "cudaSetDevice");
        return I360B_SUCCESS;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_init.load()) return I360B_SUCCESS;
    return do_initialize();
}

cudaStream_t thread_stream()
{
    unsigned gen = g_generation.load();
    if (!t_stream || t_stream_gen != gen)
    {
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        t_stream = s;
        t_stream_gen = gen;
    }
    return t_stream;
}

int dev_alloc(void** p, size_t bytes, cudaStream_t s, const char* what)
{
    *p = nullptr;
    if (bytes == 0) bytes = 256;
    if (inject_alloc_failure())
        return fail(I360B_OUT_OF_MEMORY, "%s: device allocation of %zu bytes failed (injected)", what, bytes);
    cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? I360B_OUT_OF_MEMORY : I360B_CUDA_ERROR,
                    "%s: device allocation of %zu bytes failed (%s)", what, bytes, cudaGetErrorString(e));
    }
    return I360B_SUCCESS;
}

void dev_free(void* p, cudaStream_t s)
{
    if (p) cudaFreeAsync(p, s);
}

}  // namespace i360b

using namespace i360b;

extern "C" int i360b_initialize(void)
{
    clear_error();
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_init.load()) return I360B_SUCCESS;
    return do_initialize();
}

extern "C" void i360b_shutdown(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_init.load()) return;
    cudaDeviceSynchronize();
    g_generation.fetch_add(1);
    g_init.store(false);
}

extern "C" int i360b_is_initialized(void) { return g_init.load() ? 1 : 0; }

extern "C" int i360b_debug_inject_failure(int kind, int count)
{
    clear_error();
    if (count < 0) return fail(I360B_INVALID_PARAM, "count must be >= 0.");
    if (kind == I360B_INJECT_ALLOC) g_injectAlloc.store(count);
    else if (kind == I360B_INJECT_LAUNCH) g_injectLaunch.store(count);
    else return fail(I360B_INVALID_PARAM, "Unknown injection kind %d.", kind);
    return I360B_SUCCESS;
}

extern "C" const char* i360b_get_last_error(void) { return t_err; }

extern "C" int i360b_not_supported(const char* op)
{
    return fail(I360B_NOT_SUPPORTED, "%s is not supported by the B200 backend.", op ? op : "operation");
}

extern "C" int i360b_get_gpu_info(i360b_gpu_info* out)
{
    if (!out) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    std::memset(out, 0, sizeof(*out));
    out->deviceId = -1;
    if (!g_init.load()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    cudaDeviceProp p;
    I360B_CUDA(cudaGetDeviceProperties(&p, g_device), "cudaGetDeviceProperties");
    size_t freeB = 0, totalB = 0;
    I360B_CUDA(cudaSetDevice(g_device), "cudaSetDevice");
    I360B_CUDA(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
    out->deviceId = g_device;
    std::snprintf(out->name, sizeof(out->name), "%s", p.name);
    out->totalMemory = totalB;
    out->freeMemory = freeB;
    out->computeMajor = p.major;
    out->computeMinor = p.minor;
    out->maxThreadsPerBlock = p.maxThreadsPerBlock;
    out->multiProcessorCount = p.multiProcessorCount;
    out->hasTensorCores = p.major >= 7 ? 1 : 0;
    return I360B_SUCCESS;
}
