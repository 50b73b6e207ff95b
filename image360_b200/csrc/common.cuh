// Shared device helpers and host-side runtime plumbing for the B200 render
// backend.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#include "../../include/image360_b200.h"

namespace i360b
{
// ---------------------------------------------------------------------------
// Exact FP32 arithmetic.  The reference's CPU kernels are compiled without FMA
// contraction (scalar tier and SeamBlend carry no -mfma), so every product and
// sum is rounded separately and in source order.  These wrappers keep nvcc from
// fusing multiply-adds, which would change the last bit and break parity.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// Exact integer <-> float conversions on the FMA and ALU pipes.  The
// conversion instructions (I2F/F2I) issue on the XU pipe at a fraction of the
// FMA rate, and the pixel kernels convert every sample both ways; these
// identities give the same values:
//  u2f: for 0 <= v < 2^23 the float with bits 0x4B000000 | v is 2^23 + v,
//       exactly, so subtracting 2^23 (exact) leaves v.
//  f2u_floor: for 0 <= x < 2^23, x + 2^23 rounded toward zero lies in
//       [2^23, 2^24), where floats are the integers, so it is 2^23 + floor(x)
//       and its mantissa bits are floor(x).
__device__ __forceinline__ float u2f(uint32_t v) { return __fsub_rn(__uint_as_float(0x4B000000u | v), 8388608.0f); }
__device__ __forceinline__ uint32_t f2u_floor(float x) { return __float_as_uint(__fadd_rz(x, 8388608.0f)) & 0x7FFFFFu; }

// (unsigned short)min(max(v, 0), 65535): clamp then truncate toward zero, the
// quantisation at every stage boundary of the reference (e.g.
// WarpPerspectiveKernels.h:41, BayerDemosaicKernels.h:58,73, GainColorOps.cpp:23).
__device__ __forceinline__ unsigned short clamp_trunc_u16(float v)
{
    v = v > 0.0f ? v : 0.0f;  // NaN -> 0
    v = v < 65535.0f ? v : 65535.0f;
    return static_cast<unsigned short>(f2u_floor(v));  // truncation = floor on [0, 65535]
}

// (float)clamp_trunc_u16(v) without the round trip through an integer: on
// [0, 65535], v + 2^23 rounded toward zero is 2^23 + floor(v) (the floats of
// [2^23, 2^24) are the integers) and subtracting 2^23 is exact, so this is
// u2f(clamp_trunc_u16(v)) bit for bit.
__device__ __forceinline__ float clamp_floor_u16f(float v)
{
    v = v > 0.0f ? v : 0.0f;  // NaN -> 0
    v = v < 65535.0f ? v : 65535.0f;
    return __fsub_rn(__fadd_rz(v, 8388608.0f), 8388608.0f);
}

// ApplyGain's skip rule (GainColorOps.cpp:22 and RenderExecutor.cpp:111).
__host__ __device__ __forceinline__ bool gain_is_identity(float gain)
{
    float d = gain - 1.0f;
    d = d < 0.0f ? -d : d;
    return d < 1e-6f;
}

constexpr int kMaxContributors = 32;  // RenderExecutor.cpp:15, CpuComputeBackend.cpp:143

// ---------------------------------------------------------------------------
// Host runtime (context.cu)
// ---------------------------------------------------------------------------

// Thread-local last error; returns `code` so call sites can `return fail(...)`.
int fail(int code, const char* fmt, ...);
void clear_error();
// Maps a CUDA error to a result code and records the message.
int cuda_fail(cudaError_t e, const char* what);
// Checks for a launch error of the kernel just enqueued (or an injected one).
int check_launch(const char* what);
// True when a test armed a host-side allocation failure (consumes one).
bool inject_alloc_failure();

bool initialized();
int device();
int sm_count();
// The calling thread's stream for the synchronous host-buffer API.
cudaStream_t thread_stream();
// Stream-ordered allocation from the device's pool (kept for the process life).
int dev_alloc(void** p, size_t bytes, cudaStream_t s, const char* what);
void dev_free(void* p, cudaStream_t s);

// Requires an initialised context (lazy-initialises on first use).
int ensure_ready();
// Device address of the allocation-free blend's static scratch array on the
// current device (noalloc.cu); resolved once per device.
int noalloc_scratch(void** out);

#define I360B_TRY(expr)             \
    do                              \
    {                               \
        int _rc = (expr);           \
        if (_rc != I360B_SUCCESS)   \
            return _rc;             \
    } while (0)

#define I360B_CUDA(expr, what)                        \
    do                                                \
    {                                                 \
        cudaError_t _e = (expr);                      \
        if (_e != cudaSuccess)                        \
            return ::i360b::cuda_fail(_e, what);      \
    } while (0)

// Kernel launchers shared between translation units (all stream-ordered).
int launch_demosaic(const unsigned short* cfa, int w, int h, unsigned short black, const float* camMul,
                    const float* rgbCam, uint32_t filters, unsigned short* out, cudaStream_t s);
int launch_warp(const unsigned short* src, int sw, int sh, unsigned short* dst, int dw, int dh, const float* H,
                int offX, int offY, float gain, cudaStream_t s);
int launch_median(const unsigned short* const* inputs, int n, unsigned short* out, int w, int h, float sigma,
                  cudaStream_t s);
int launch_warp_median(const unsigned short* const* frames, int n, int sw, int sh, const float* H, unsigned short* out,
                       int dw, int dh, int offX, int offY, float sigma, cudaStream_t s);
int launch_gain(unsigned short* data, long long n, float gain, cudaStream_t s);
// Lab statistics / Reinhard transfer / frame-set colour correction (color.cu).
int launch_lab_stats(const unsigned short* const* dImgs, const int* w, const int* h, int n, double* dStats,
                     cudaStream_t s);
int launch_reinhard(unsigned short* const* dImgs, const int* w, const int* h, int n, const double* dSrcStats,
                    const double* dRefStats, cudaStream_t s);
int launch_color_correct(unsigned short* const* dImgs, const int* w, const int* h, int n, int refIndex,
                         double* dStats, cudaStream_t s);
int launch_blend_chunk(const unsigned short* const* warped, int k, int w, int h, int bands, unsigned short* out,
                       cudaStream_t s);
// The same blend with all device scratch carved from a caller-provided buffer
// (no allocation); synchronous on `s`.
int launch_blend_chunk_in(void* arena, size_t arenaBytes, const unsigned short* const* warped, int k, int w, int h,
                          int bands, unsigned short* out, cudaStream_t s);
}  // namespace i360b
