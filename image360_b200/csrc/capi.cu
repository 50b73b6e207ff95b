// C-ABI entry points of the IComputeBackend operations: argument checks with
// the CPU backend's messages and result codes (CpuComputeBackend.cpp:112-193),
// then host->device copies, the kernel, and the device->host copy on the
// calling thread's stream.
#include "common.cuh"

#include <vector>

using namespace i360b;

namespace
{
// RAII for stream-ordered scratch.
struct DevBuf
{
    void* p = nullptr;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { dev_free(p, s); }
    int alloc(size_t bytes, cudaStream_t st, const char* what)
    {
        s = st;
        return dev_alloc(&p, bytes, st, what);
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

int require_init()
{
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    return ensure_ready();
}

int sync(cudaStream_t s, const char* what)
{
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, what);
    return I360B_SUCCESS;
}

cudaStream_t get_stream(int* rc)
{
    cudaStream_t s = thread_stream();
    *rc = s ? I360B_SUCCESS : fail(I360B_CUDA_ERROR, "Could not create a CUDA stream for this thread.");
    return s;
}
}  // namespace

extern "C" int i360b_warp_perspective(const unsigned short* srcData, int srcW, int srcH, unsigned short* dstData,
                                      int dstW, int dstH, const float* homography, int offsetX, int offsetY)
{
    clear_error();
    I360B_TRY(require_init());
    if (!srcData || !dstData || !homography) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (srcW <= 0 || srcH <= 0 || dstW <= 0 || dstH <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    int rc;
    cudaStream_t s = get_stream(&rc);
    I360B_TRY(rc);
    size_t sb = (size_t)srcW * srcH * 6, db = (size_t)dstW * dstH * 6;
    DevBuf dS, dD;
    I360B_TRY(dS.alloc(sb, s, "WarpPerspective"));
    I360B_TRY(dD.alloc(db, s, "WarpPerspective"));
    I360B_CUDA(cudaMemcpyAsync(dS.p, srcData, sb, cudaMemcpyHostToDevice, s), "WarpPerspective upload");
    I360B_TRY(launch_warp(dS.as<unsigned short>(), srcW, srcH, dD.as<unsigned short>(), dstW, dstH, homography, offsetX,
                          offsetY, 1.0f, s));
    I360B_CUDA(cudaMemcpyAsync(dstData, dD.p, db, cudaMemcpyDeviceToHost, s), "WarpPerspective download");
    return sync(s, "WarpPerspective");
}

extern "C" int i360b_median_stack(const unsigned short* const* inputs, int numInputs, unsigned short* output,
                                  int width, int height, float sigmaThreshold)
{
    clear_error();
    I360B_TRY(require_init());
    if (!inputs || !output) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (numInputs <= 0 || numInputs > 32) return fail(I360B_INVALID_PARAM, "numInputs must be 1-32.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    for (int i = 0; i < numInputs; ++i)
        if (!inputs[i]) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    int rc;
    cudaStream_t s = get_stream(&rc);
    I360B_TRY(rc);
    size_t plane = (size_t)width * height * 3 * 2;
    DevBuf dIn, dOut;
    I360B_TRY(dIn.alloc(plane * numInputs, s, "MedianStack"));
    I360B_TRY(dOut.alloc(plane, s, "MedianStack"));
    const unsigned short* ptrs[kMaxContributors];
    for (int i = 0; i < numInputs; ++i)
    {
        unsigned short* d = dIn.as<unsigned short>() + (size_t)i * plane / 2;
        I360B_CUDA(cudaMemcpyAsync(d, inputs[i], plane, cudaMemcpyHostToDevice, s), "MedianStack upload");
        ptrs[i] = d;
    }
    I360B_TRY(launch_median(ptrs, numInputs, dOut.as<unsigned short>(), width, height, sigmaThreshold, s));
    I360B_CUDA(cudaMemcpyAsync(output, dOut.p, plane, cudaMemcpyDeviceToHost, s), "MedianStack download");
    return sync(s, "MedianStack");
}

extern "C" int i360b_apply_gain(unsigned short* data, int numPixels, float gain)
{
    clear_error();
    I360B_TRY(require_init());
    if (!data) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (numPixels <= 0) return fail(I360B_INVALID_PARAM, "Invalid pixel count.");
    if (gain_is_identity(gain)) return I360B_SUCCESS;  // GainColorOps.cpp:22
    int rc;
    cudaStream_t s = get_stream(&rc);
    I360B_TRY(rc);
    size_t b = (size_t)numPixels * 2;
    DevBuf d;
    I360B_TRY(d.alloc(b, s, "ApplyGain"));
    I360B_CUDA(cudaMemcpyAsync(d.p, data, b, cudaMemcpyHostToDevice, s), "ApplyGain upload");
    I360B_TRY(launch_gain(d.as<unsigned short>(), numPixels, gain, s));
    I360B_CUDA(cudaMemcpyAsync(data, d.p, b, cudaMemcpyDeviceToHost, s), "ApplyGain download");
    return sync(s, "ApplyGain");
}

extern "C" int i360b_compute_lab_stats(const unsigned short* rgb, int width, int height, double outMean[3],
                                       double outStd[3])
{
    clear_error();
    I360B_TRY(require_init());
    if (!rgb || !outMean || !outStd) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    int rc;
    cudaStream_t s = get_stream(&rc);
    I360B_TRY(rc);
    size_t b = (size_t)width * height * 6;
    DevBuf d, st;
    I360B_TRY(d.alloc(b, s, "ComputeLabStats"));
    I360B_TRY(st.alloc(6 * sizeof(double), s, "ComputeLabStats"));
    I360B_CUDA(cudaMemcpyAsync(d.p, rgb, b, cudaMemcpyHostToDevice, s), "ComputeLabStats upload");
    const unsigned short* img = d.as<unsigned short>();
    I360B_TRY(launch_lab_stats(&img, &width, &height, 1, st.as<double>(), s));
    double h[6];
    I360B_CUDA(cudaMemcpyAsync(h, st.p, sizeof(h), cudaMemcpyDeviceToHost, s), "ComputeLabStats download");
    I360B_TRY(sync(s, "ComputeLabStats"));
    for (int c = 0; c < 3; ++c)
    {
        outMean[c] = h[c];
        outStd[c] = h[3 + c];
    }
    return I360B_SUCCESS;
}

extern "C" int i360b_apply_reinhard_color_transfer(unsigned short* rgbInOut, int width, int height,
                                                   const double srcMean[3], const double srcStd[3],
                                                   const double refMean[3], const double refStd[3])
{
    clear_error();
    I360B_TRY(require_init());
    if (!rgbInOut || !srcMean || !srcStd || !refMean || !refStd)
        return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    int rc;
    cudaStream_t s = get_stream(&rc);
    I360B_TRY(rc);
    size_t b = (size_t)width * height * 6;
    DevBuf d, st;
    I360B_TRY(d.alloc(b, s, "ApplyReinhardColorTransfer"));
    I360B_TRY(st.alloc(12 * sizeof(double), s, "ApplyReinhardColorTransfer"));
    const double h[12] = {srcMean[0], srcMean[1], srcMean[2], srcStd[0], srcStd[1], srcStd[2],
                          refMean[0], refMean[1], refMean[2], refStd[0], refStd[1], refStd[2]};
    I360B_CUDA(cudaMemcpyAsync(st.p, h, sizeof(h), cudaMemcpyHostToDevice, s), "ApplyReinhardColorTransfer upload");
    I360B_CUDA(cudaMemcpyAsync(d.p, rgbInOut, b, cudaMemcpyHostToDevice, s), "ApplyReinhardColorTransfer upload");
    unsigned short* img = d.as<unsigned short>();
    I360B_TRY(launch_reinhard(&img, &width, &height, 1, st.as<double>(), st.as<double>() + 6, s));
    I360B_CUDA(cudaMemcpyAsync(rgbInOut, d.p, b, cudaMemcpyDeviceToHost, s), "ApplyReinhardColorTransfer download");
    return sync(s, "ApplyReinhardColorTransfer");
}

extern "C" int i360b_demosaic_bayer(const unsigned short* cfaData, int width, int height, unsigned short blackLevel,
                                    const float camMul[4], const float rgbCam[12], uint32_t filters,
                                    unsigned short* rgbOut)
{
    clear_error();
    I360B_TRY(require_init());
    if (!cfaData || !camMul || !rgbCam || !rgbOut) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    int rc;
    cudaStream_t s = get_stream(&rc);
    I360B_TRY(rc);
    size_t cb = (size_t)width * height * 2, ob = cb * 3;
    DevBuf dC, dO;
    I360B_TRY(dC.alloc(cb, s, "DemosaicBayer"));
    I360B_TRY(dO.alloc(ob, s, "DemosaicBayer"));
    I360B_CUDA(cudaMemcpyAsync(dC.p, cfaData, cb, cudaMemcpyHostToDevice, s), "DemosaicBayer upload");
    I360B_TRY(launch_demosaic(dC.as<unsigned short>(), width, height, blackLevel, camMul, rgbCam, filters,
                              dO.as<unsigned short>(), s));
    I360B_CUDA(cudaMemcpyAsync(rgbOut, dO.p, ob, cudaMemcpyDeviceToHost, s), "DemosaicBayer download");
    return sync(s, "DemosaicBayer");
}

extern "C" int i360b_blend_chunk_contributors(const unsigned short* const* warpedBuffers, int numContributors,
                                              int width, int height, int numBands, unsigned short* outResult)
{
    clear_error();
    I360B_TRY(require_init());
    if (!outResult || (numContributors > 0 && !warpedBuffers)) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    if (numContributors < 0 || numContributors > 127)
        return fail(I360B_INVALID_PARAM, "numContributors must be 0-127.");
    if (numBands < 1) return fail(I360B_INVALID_PARAM, "numBands must be >= 1.");
    for (int i = 0; i < numContributors; ++i)
        if (!warpedBuffers[i]) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    int rc;
    cudaStream_t s = get_stream(&rc);
    I360B_TRY(rc);
    size_t plane = (size_t)width * height * 6;
    DevBuf dIn, dOut;
    I360B_TRY(dIn.alloc(plane * (numContributors > 0 ? numContributors : 1), s, "BlendChunkContributors"));
    I360B_TRY(dOut.alloc(plane, s, "BlendChunkContributors"));
    std::vector<const unsigned short*> ptrs(numContributors);
    for (int i = 0; i < numContributors; ++i)
    {
        unsigned short* d = dIn.as<unsigned short>() + (size_t)i * plane / 2;
        I360B_CUDA(cudaMemcpyAsync(d, warpedBuffers[i], plane, cudaMemcpyHostToDevice, s), "BlendChunkContributors upload");
        ptrs[i] = d;
    }
    I360B_TRY(launch_blend_chunk(ptrs.data(), numContributors, width, height, numBands, dOut.as<unsigned short>(), s));
    I360B_CUDA(cudaMemcpyAsync(outResult, dOut.p, plane, cudaMemcpyDeviceToHost, s), "BlendChunkContributors download");
    return sync(s, "BlendChunkContributors");
}

// ---- device-resident launchers --------------------------------------------

extern "C" int i360b_launch_demosaic(const unsigned short* dCfa, int width, int height, unsigned short blackLevel,
                                     const float camMul[4], const float rgbCam[12], uint32_t filters,
                                     unsigned short* dRgbOut, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    if (!dCfa || !camMul || !rgbCam || !dRgbOut) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    return launch_demosaic(dCfa, width, height, blackLevel, camMul, rgbCam, filters, dRgbOut,
                           static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_launch_warp(const unsigned short* dSrc, int srcW, int srcH, unsigned short* dDst, int dstW,
                                 int dstH, const float* homography, int offsetX, int offsetY, float gain, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    if (!dSrc || !dDst || !homography) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (srcW <= 0 || srcH <= 0 || dstW <= 0 || dstH <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    return launch_warp(dSrc, srcW, srcH, dDst, dstW, dstH, homography, offsetX, offsetY, gain,
                       static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_launch_median(const unsigned short* const* dInputs, int numInputs, unsigned short* dOutput,
                                   int width, int height, float sigmaThreshold, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    if (!dInputs || !dOutput) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (numInputs <= 0 || numInputs > 32) return fail(I360B_INVALID_PARAM, "numInputs must be 1-32.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    for (int i = 0; i < numInputs; ++i)
        if (!dInputs[i]) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    return launch_median(dInputs, numInputs, dOutput, width, height, sigmaThreshold, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_launch_warp_median(const unsigned short* const* dFrames, int numFrames, int srcW, int srcH,
                                        const float* homographies, unsigned short* dOutput, int dstW, int dstH,
                                        int offsetX, int offsetY, float sigmaThreshold, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    if (!dFrames || !dOutput || !homographies) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (numFrames <= 0 || numFrames > 32) return fail(I360B_INVALID_PARAM, "numInputs must be 1-32.");
    if (srcW <= 0 || srcH <= 0 || dstW <= 0 || dstH <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    for (int i = 0; i < numFrames; ++i)
        if (!dFrames[i]) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    return launch_warp_median(dFrames, numFrames, srcW, srcH, homographies, dOutput, dstW, dstH, offsetX, offsetY,
                              sigmaThreshold, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_launch_gain(unsigned short* dData, int numValues, float gain, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    if (!dData) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (numValues <= 0) return fail(I360B_INVALID_PARAM, "Invalid pixel count.");
    return launch_gain(dData, numValues, gain, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_launch_lab_stats(const unsigned short* const* dImages, const int* widths, const int* heights,
                                      int n, double* dStats, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    return launch_lab_stats(dImages, widths, heights, n, dStats, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_launch_reinhard(unsigned short* const* dImages, const int* widths, const int* heights, int n,
                                     const double* dSrcStats, const double* dRefStats, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    return launch_reinhard(dImages, widths, heights, n, dSrcStats, dRefStats, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_launch_color_correct(unsigned short* const* dImages, const int* widths, const int* heights,
                                          int n, int refIndex, double* dStats, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    return launch_color_correct(dImages, widths, heights, n, refIndex, dStats, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_launch_blend(const unsigned short* const* dWarped, int numContributors, int width, int height,
                                  int numBands, unsigned short* dOut, void* stream)
{
    clear_error();
    I360B_TRY(require_init());
    if (!dOut || (numContributors > 0 && !dWarped)) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    if (numContributors < 0 || numContributors > 127) return fail(I360B_INVALID_PARAM, "numContributors must be 0-127.");
    if (numBands < 1) return fail(I360B_INVALID_PARAM, "numBands must be >= 1.");
    for (int i = 0; i < numContributors; ++i)
        if (!dWarped[i]) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    return launch_blend_chunk(dWarped, numContributors, width, height, numBands, dOut, static_cast<cudaStream_t>(stream));
}
