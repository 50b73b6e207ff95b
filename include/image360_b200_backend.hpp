// B200ComputeBackend: the WindowsApp::Compute::IComputeBackend implementation
// (WindowsApp.Compute/HeaderFiles/IComputeBackend.h:16-169) over the C-ABI in
// image360_b200.h, plus the IRenderBlendBackend extension that exposes the
// seam blend and the batched device-resident tile render.
//
// Header-only.  Compile it inside the reference project, with
// WindowsApp.Compute/HeaderFiles on the include path, and link
// libimage360_b200.so.  ComputeBackendFactory then selects it like the other
// backends once a TryB200 branch names it (ComputeBackendFactory.cpp:108-135).
//
// Semantics follow the reference backends: Initialize() before use, every
// operation returns a ComputeResult, GetLastError() describes the last failure
// of the calling thread.  Host-pointer operations are synchronous.  The eight
// operations outside the render path return NOT_SUPPORTED, the way
// CudaPipeline reports CPU-only operations (CudaPipeline.cpp:794-840).
#pragma once

#include "IComputeBackend.h"
#include "image360_b200.h"

#include <cstring>

namespace WindowsApp { namespace Compute
{
    // Render-path extension with no IComputeBackend counterpart.
    // RenderExecutor would dynamic_cast its backend to this to hand the
    // blend, or a whole panorama's tiles, to the GPU.
    class IRenderBlendBackend
    {
    public:
        virtual ~IRenderBlendBackend() = default;

        // Kernels::SeamBlend::BlendChunkContributors (SeamBlendKernels.h:91)
        // with the band count of Detail::MultiBandCompose (5 = default).
        virtual ComputeResult BlendChunkContributors(
            const unsigned short* const* warpedBuffers, int numContributors,
            int width, int height, int numBands, unsigned short* outResult) = 0;

        // Device-resident render of many uneven tiles (see image360_b200.h).
        virtual ComputeResult CreateRenderPlan(
            const i360b_frame* frames, int numFrames, const i360b_tile* tiles, int numTiles,
            const int* contributors, int numBands, int coordMode, i360b_render_plan** outPlan) = 0;
        virtual ComputeResult ExecuteRenderPlan(i360b_render_plan* plan, void* stream) = 0;
        virtual ComputeResult WaitRenderPlan(i360b_render_plan* plan, void* stream) = 0;
        virtual void DestroyRenderPlan(i360b_render_plan* plan) = 0;
    };

    class B200ComputeBackend final : public IComputeBackend, public IRenderBlendBackend
    {
    public:
        B200ComputeBackend() = default;
        ~B200ComputeBackend() override = default;

        ComputeResult Initialize() override { return R(i360b_initialize()); }
        void Shutdown() override { i360b_shutdown(); }
        bool IsInitialized() const override { return i360b_is_initialized() != 0; }

        GpuInfo GetGpuInfo() const override
        {
            GpuInfo info;
            i360b_gpu_info c{};
            if (i360b_get_gpu_info(&c) == I360B_SUCCESS)
            {
                info.deviceId = c.deviceId;
                std::memcpy(info.name, c.name, sizeof(info.name));
                info.totalMemory = c.totalMemory;
                info.freeMemory = c.freeMemory;
                info.computeMajor = c.computeMajor;
                info.computeMinor = c.computeMinor;
                info.maxThreadsPerBlock = c.maxThreadsPerBlock;
                info.multiProcessorCount = c.multiProcessorCount;
                info.hasTensorCores = c.hasTensorCores != 0;
            }
            return info;
        }

        const char* GetLastError() const override { return i360b_get_last_error(); }

        ComputeResult WarpPerspective(
            const unsigned short* srcData, int srcW, int srcH,
            unsigned short* dstData, int dstW, int dstH,
            const float* homography, int offsetX, int offsetY) override
        {
            return R(i360b_warp_perspective(srcData, srcW, srcH, dstData, dstW, dstH, homography, offsetX, offsetY));
        }

        ComputeResult MedianStack(
            const unsigned short** inputs, int numInputs,
            unsigned short* output, int width, int height,
            float sigmaThreshold = 2.0f) override
        {
            return R(i360b_median_stack(inputs, numInputs, output, width, height, sigmaThreshold));
        }

        ComputeResult ApplyGain(unsigned short* data, int numPixels, float gain) override
        {
            return R(i360b_apply_gain(data, numPixels, gain));
        }

        ComputeResult DemosaicBayer(
            const unsigned short* cfaData, int width, int height,
            unsigned short blackLevel, const float camMul[4], const float rgbCam[3][4],
            uint32_t filters, unsigned short* rgbOut) override
        {
            return R(i360b_demosaic_bayer(cfaData, width, height, blackLevel, camMul,
                                          rgbCam ? &rgbCam[0][0] : nullptr, filters, rgbOut));
        }

        ComputeResult DetectAndDescribeFeatures(const unsigned char*, int, int, FeaturePoint*, BriefDescriptor*,
                                                int*, int) override
        {
            return R(i360b_not_supported("DetectAndDescribeFeatures"));
        }
        ComputeResult MatchFeatures(const BriefDescriptor*, int, const BriefDescriptor*, int, MatchResult*, int*, int,
                                    float = 0.75f) override
        {
            return R(i360b_not_supported("MatchFeatures"));
        }
        ComputeResult ComputeLabStats(const unsigned short* rgb, int width, int height, double outMean[3],
                                      double outStd[3]) override
        {
            return R(i360b_compute_lab_stats(rgb, width, height, outMean, outStd));
        }
        ComputeResult ApplyReinhardColorTransfer(unsigned short* rgbInOut, int width, int height,
                                                 const double srcMean[3], const double srcStd[3],
                                                 const double refMean[3], const double refStd[3]) override
        {
            return R(i360b_apply_reinhard_color_transfer(rgbInOut, width, height, srcMean, srcStd, refMean,
                                                         refStd));
        }
        ComputeResult BlockMatchAlign(const unsigned short*, const unsigned short*, int, int, int, int, TileOffset*,
                                      int, int) override
        {
            return R(i360b_not_supported("BlockMatchAlign"));
        }
        ComputeResult RobustMergeAccumulate(const unsigned short* const*, int, const TileOffset* const*, int, int, int,
                                            int, int, float, unsigned short*) override
        {
            return R(i360b_not_supported("RobustMergeAccumulate"));
        }
        ComputeResult TileFftMerge(const unsigned short* const*, int, const TileOffset* const*, int, int, int, int,
                                   int, float, unsigned short*) override
        {
            return R(i360b_not_supported("TileFftMerge"));
        }
        ComputeResult StructureTensorKernelRegression(const unsigned short* const*, int, const TileOffsetF* const*,
                                                      int, int, int, int, int, int, float, unsigned short*) override
        {
            return R(i360b_not_supported("StructureTensorKernelRegression"));
        }

        // IRenderBlendBackend
        ComputeResult BlendChunkContributors(const unsigned short* const* warpedBuffers, int numContributors,
                                             int width, int height, int numBands, unsigned short* outResult) override
        {
            return R(i360b_blend_chunk_contributors(warpedBuffers, numContributors, width, height, numBands, outResult));
        }
        ComputeResult CreateRenderPlan(const i360b_frame* frames, int numFrames, const i360b_tile* tiles, int numTiles,
                                       const int* contributors, int numBands, int coordMode,
                                       i360b_render_plan** outPlan) override
        {
            return R(i360b_render_plan_create(frames, numFrames, tiles, numTiles, contributors, numBands, coordMode,
                                              outPlan));
        }
        ComputeResult ExecuteRenderPlan(i360b_render_plan* plan, void* stream) override
        {
            return R(i360b_render_plan_execute(plan, stream));
        }
        ComputeResult WaitRenderPlan(i360b_render_plan* plan, void* stream) override
        {
            return R(i360b_render_plan_wait(plan, stream));
        }
        void DestroyRenderPlan(i360b_render_plan* plan) override { i360b_render_plan_destroy(plan); }

    private:
        static ComputeResult R(int code) { return static_cast<ComputeResult>(code); }
    };
}}
