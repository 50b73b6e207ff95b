// Test infrastructure only: a C-ABI shim over the reference's own CPU code
// (thnak/Image360, WindowsApp.Core), compiled from the reference sources in
// place by oracle/Makefile into oracle/_ref/libi360ref.so.  Nothing in the
// product links or loads this; the tests use it to pin the C restatement in
// oracle/i360_oracle.c, the golden-fixture script uses it to produce golden
// vectors, and bench.py's CPU-baseline leg times it.
//
// Every function forwards to the reference implementation named beside it;
// no arithmetic happens here except the task loop of ref_render_tiles, which
// drives the reference kernels the way RenderExecutor::Execute does
// (WindowsApp.Core/SourceFiles/RenderExecutor.cpp:70-140) with the reference's
// CPU-backend concurrency model (hardware_concurrency()-1 single-threaded
// tasks, WindowsApp/WindowsApp/ComputeBackendFactory.cpp:99-100).

#include "HeaderFiles/CpuComputeBackend.h"
#include "HeaderFiles/CpuSimdDetect.h"
#include "HeaderFiles/MedianStackKernels.h"
#include "HeaderFiles/WarpPerspectiveKernels.h"
#include "HeaderFiles/BayerDemosaicKernels.h"
#include "HeaderFiles/GainColorOps.h"
#include "HeaderFiles/HomographyMath.h"
#include "HeaderFiles/SeamBlendKernels.h"
#include "HeaderFiles/OverlapCulling.h"
#include "HeaderFiles/PanoramaExporter.h"
#include "HeaderFiles/StorageEngine.h"
#include "HeaderFiles/TextEncoding.h"
#include "HeaderFiles/Tiff16Writer.h"

#include <atomic>
#include <memory>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

using namespace WindowsApp::Core;

namespace WindowsApp::Core
{
void RefStubAddRenderTask(const std::string& chunkId, int64_t blobId);  // ref_project_stub.cpp
}

namespace
{
// An image codec that keeps the RGB8 image it is asked to encode (the
// preview composite) and returns it as the "encoded" bytes.
class CapturingCodec final : public WindowsApp::Compute::IImageCodec
{
public:
    std::vector<unsigned char> rgb;
    int width = 0, height = 0;
    WindowsApp::Compute::ComputeResult Initialize() override { return WindowsApp::Compute::ComputeResult::SUCCESS; }
    void Shutdown() override {}
    WindowsApp::Compute::ComputeResult Decode(const unsigned char*, size_t, unsigned char**, int*, int*) override
    {
        return WindowsApp::Compute::ComputeResult::NOT_SUPPORTED;
    }
    void FreeDecoded(unsigned char*) override {}
    WindowsApp::Compute::ComputeResult Encode(const unsigned char* data, int w, int h, int, std::vector<unsigned char>& out) override
    {
        width = w;
        height = h;
        rgb.assign(data, data + static_cast<size_t>(w) * h * 3);
        out = rgb;
        return WindowsApp::Compute::ComputeResult::SUCCESS;
    }
    const char* GetLastError() const override { return ""; }
};
}  // namespace
namespace SB = WindowsApp::Core::Kernels::SeamBlend;
using WindowsApp::Compute::ComputeResult;

namespace
{
    // rgbCam arrives as 12 floats, row-major 3x4.
    void Unflatten(const float* flat, float out[3][4])
    {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) out[r][c] = flat[r * 4 + c];
    }

    // Same steps as SB::BlendChunkContributors (SeamBlend.cpp:549-587) with the
    // band count exposed, the way Detail::MultiBandCompose is public for it
    // (SeamBlendKernels.h:75-79).
    void BlendWithBands(const std::vector<const unsigned short*>& bufs, int w, int h, int bands,
                        std::vector<unsigned short>& out)
    {
        size_t count = static_cast<size_t>(w) * h;
        out.assign(count * 3, 0);
        int k = static_cast<int>(bufs.size());
        if (k == 0) return;
        std::vector<std::vector<unsigned char>> covered(k);
        std::vector<std::vector<float>> dist(k);
        std::vector<SB::Detail::BBox> boxes(k);
        for (int i = 0; i < k; ++i)
        {
            covered[i].assign(count, 0);
            const unsigned short* b = bufs[i];
            for (size_t p = 0; p < count; ++p)
                covered[i][p] = (b[p * 3] != 0 || b[p * 3 + 1] != 0 || b[p * 3 + 2] != 0) ? 1 : 0;
            SB::Detail::ComputeCoverageDistance(covered[i], w, h, dist[i]);
            boxes[i] = SB::Detail::ComputeCoverageBBox(covered[i], w, h);
        }
        std::vector<int> owner;
        SB::Detail::ComputeOwnership(dist, w, h, owner);
        for (int i = 0; i < k; ++i)
        {
            if (!boxes[i].valid) continue;
            for (int j = i + 1; j < k; ++j)
            {
                if (!boxes[j].valid) continue;
                SB::Detail::BBox ov;
                if (!SB::Detail::IntersectBBox(boxes[i], boxes[j], ov)) continue;
                SB::Detail::RefineSeamDP(bufs[i], bufs[j], dist[i], dist[j], w, h, i, j, boxes[i], boxes[j], ov, owner);
            }
        }
        SB::Detail::MultiBandCompose(bufs, dist, owner, w, h, bands, out);
    }
}

extern "C"
{
    // CpuSimdDetect.cpp:110-118.  0 = scalar, 1 = AVX2, 2 = AVX-512.
    int ref_simd_tier()
    {
        switch (DetectCpuSimdTier())
        {
        case SimdTier::Avx512: return 2;
        case SimdTier::Avx2: return 1;
        default: return 0;
        }
    }

    // Kernels::{Scalar,Avx2,Avx512}::DemosaicBayer (BayerDemosaic_*.cpp).
    void ref_demosaic(int tier, const uint16_t* cfa, int w, int h, uint16_t black,
                      const float* camMul, const float* rgbCamFlat, uint32_t filters, uint16_t* out)
    {
        float rgbCam[3][4];
        Unflatten(rgbCamFlat, rgbCam);
        if (tier == 2) Kernels::Avx512::DemosaicBayer(cfa, w, h, black, camMul, rgbCam, filters, out);
        else if (tier == 1) Kernels::Avx2::DemosaicBayer(cfa, w, h, black, camMul, rgbCam, filters, out);
        else Kernels::Scalar::DemosaicBayer(cfa, w, h, black, camMul, rgbCam, filters, out);
    }

    // Kernels::{Scalar,Avx2,Avx512}::WarpPerspective (WarpPerspective_*.cpp).
    void ref_warp(int tier, const uint16_t* src, int sw, int sh, uint16_t* dst, int dw, int dh,
                  const float* invH, int offX, int offY)
    {
        if (tier == 2) Kernels::Avx512::WarpPerspective(src, sw, sh, dst, dw, dh, invH, offX, offY);
        else if (tier == 1) Kernels::Avx2::WarpPerspective(src, sw, sh, dst, dw, dh, invH, offX, offY);
        else Kernels::Scalar::WarpPerspective(src, sw, sh, dst, dw, dh, invH, offX, offY);
    }

    // Kernels::{Scalar,Avx2,Avx512}::MedianStack (MedianStack_*.cpp).
    void ref_median(int tier, const uint16_t** inputs, int n, uint16_t* out, int w, int h, float sigma)
    {
        if (tier == 2) Kernels::Avx512::MedianStack(inputs, n, out, w, h, sigma);
        else if (tier == 1) Kernels::Avx2::MedianStack(inputs, n, out, w, h, sigma);
        else Kernels::Scalar::MedianStack(inputs, n, out, w, h, sigma);
    }

    // ApplyGainCpu (GainColorOps.cpp:16-26).
    void ref_gain(uint16_t* data, int n, float gain) { ApplyGainCpu(data, n, gain); }

    // OverlapCulling.cpp:36-71.
    int ref_image_overlaps_chunk(const float* h9, int iw, int ih, int cx, int cy, int cw, int ch)
    {
        Homography h;
        for (int i = 0; i < 9; ++i) h.h[i] = h9[i];
        ChunkModel c;
        c.x_offset = cx;
        c.y_offset = cy;
        c.width = cw;
        c.height = ch;
        return ImageOverlapsChunk(h, iw, ih, c) ? 1 : 0;
    }

    // OverlapCulling.cpp:73-115 with files that cannot be opened (the image
    // loader is stubbed in ref_loader_stub.cpp): writes the ids returned.
    int ref_find_overlapping_unopenable(int n, int* idsOut)
    {
        ChunkModel c;
        std::vector<InputImageModel> images(n);
        for (int i = 0; i < n; ++i)
        {
            images[i].id = 100 + i;
            images[i].file_path = L"/nonexistent/frame.dng";
        }
        auto r = FindOverlappingImages(c, images);
        for (size_t i = 0; i < r.size(); ++i) idsOut[i] = r[i];
        return static_cast<int>(r.size());
    }

    // PanoramaExporter.cpp:34-114 run on a project whose chunk grid is
    // totalW x totalH in chunkSize tiles (ProjectManager.cpp:260-281 order);
    // chunk c's render output is tiles[c] (RGB48, the chunk's size), or no
    // render task when tiles[c] is null.  Each output goes through the
    // reference's StorageEngine::WritePixelBuffer into shard files under
    // `dir` (a file prefix); the preview composite (RGB8) is captured from the
    // codec into rgbOut (capacity bytes).  Returns 1 on success and writes
    // the composite size; the framed blob of chunk `frameChunk` (or none when
    // -1) is copied to frameOut (frameCapacity bytes, size to *frameBytes).
    int ref_export_preview(const uint16_t* const* tiles, int totalW, int totalH, int chunkSize, int maxDimension,
                           const char* dir, uint8_t* rgbOut, long long capacity, int* outW, int* outH,
                           int frameChunk, uint8_t* frameOut, long long frameCapacity, long long* frameBytes)
    {
        ProjectManager pm;
        pm.CreateProject(L"", totalW, totalH, chunkSize);
        StorageEngine se;
        if (!se.Open(Utf8ToWide(dir), L"ref", pm)) return 0;
        int c = 0;
        for (const auto& chunk : pm.GetChunks())
        {
            if (tiles[c])
            {
                PixelBuffer pb;
                pb.width = chunk.width;
                pb.height = chunk.height;
                pb.data.assign(tiles[c], tiles[c] + static_cast<size_t>(chunk.width) * chunk.height * 3);
                auto id = se.WritePixelBuffer(pb, "rendered_chunk_rgb48");  // RenderExecutor.cpp:142
                if (!id.has_value()) return 0;
                RefStubAddRenderTask(chunk.id, *id);
                if (c == frameChunk && frameOut && frameBytes)
                {
                    auto blob = se.ReadBlob(*id);
                    if (!blob.has_value() || static_cast<long long>(blob->size()) > frameCapacity) return 0;
                    std::memcpy(frameOut, blob->data(), blob->size());
                    *frameBytes = static_cast<long long>(blob->size());
                }
            }
            ++c;
        }
        auto codec = std::make_shared<CapturingCodec>();
        PanoramaExporter ex(pm, se, codec);
        std::string preview = std::string(dir) + "_preview.bin";
        if (!ex.ExportPreviewJpeg(Utf8ToWide(preview), maxDimension, 90)) return 0;
        se.Close();
        if (static_cast<long long>(codec->rgb.size()) > capacity) return 0;
        std::memcpy(rgbOut, codec->rgb.data(), codec->rgb.size());
        *outW = codec->width;
        *outH = codec->height;
        return 1;
    }

    // Tiff16Writer.cpp:40-97.
    int ref_write_tiff16(const char* path, const uint16_t* data, int w, int h)
    {
        return WriteTiff16RGB(Utf8ToWide(path), data, w, h) ? 1 : 0;
    }

    // PanoramaExporter.cpp:9-24.
    float ref_export_scale(int totalW, int totalH, int maxDimension)
    {
        return ComputeExportScale(totalW, totalH, maxDimension);
    }
    void ref_chunk_placement(int x, int y, int w, int h, float scale, int* out4)
    {
        ChunkModel c;
        c.x_offset = x;
        c.y_offset = y;
        c.width = w;
        c.height = h;
        ChunkPlacement p = ComputeChunkPlacement(c, scale);
        out4[0] = p.destX;
        out4[1] = p.destY;
        out4[2] = p.destW;
        out4[3] = p.destH;
    }

    // GainColorOps.cpp:103-130 / 132-156.
    void ref_lab_stats(const uint16_t* rgb, int w, int h, double* mean, double* sd)
    {
        ComputeLabStatsCpu(rgb, w, h, mean, sd);
    }
    void ref_reinhard(uint16_t* rgb, int w, int h, const double* sm, const double* ss, const double* rm,
                      const double* rs)
    {
        ApplyReinhardColorTransferCpu(rgb, w, h, sm, ss, rm, rs);
    }

    // InvertHomography3x3 (HomographyMath.cpp:94-116).
    int ref_invert_h(const float* h, float* out) { return InvertHomography3x3(h, out) ? 1 : 0; }

    // CpuComputeBackend facade (CpuComputeBackend.cpp:70-193): argument
    // checks and error strings.
    void* ref_backend_new() { return new CpuComputeBackend(); }
    void ref_backend_free(void* b) { delete static_cast<CpuComputeBackend*>(b); }
    int ref_backend_init(void* b) { return static_cast<int>(static_cast<CpuComputeBackend*>(b)->Initialize()); }
    const char* ref_backend_last_error(void* b) { return static_cast<CpuComputeBackend*>(b)->GetLastError(); }
    int ref_backend_warp(void* b, const uint16_t* src, int sw, int sh, uint16_t* dst, int dw, int dh,
                         const float* H, int offX, int offY)
    {
        return static_cast<int>(static_cast<CpuComputeBackend*>(b)->WarpPerspective(src, sw, sh, dst, dw, dh, H, offX, offY));
    }
    int ref_backend_median(void* b, const uint16_t** in, int n, uint16_t* out, int w, int h, float sigma)
    {
        return static_cast<int>(static_cast<CpuComputeBackend*>(b)->MedianStack(in, n, out, w, h, sigma));
    }
    int ref_backend_gain(void* b, uint16_t* d, int n, float g)
    {
        return static_cast<int>(static_cast<CpuComputeBackend*>(b)->ApplyGain(d, n, g));
    }
    int ref_backend_demosaic(void* b, const uint16_t* cfa, int w, int h, uint16_t black,
                             const float* camMul, const float* rgbCamFlat, uint32_t filters, uint16_t* out)
    {
        float rgbCam[3][4];
        const float (*cam)[4] = nullptr;
        if (rgbCamFlat) { Unflatten(rgbCamFlat, rgbCam); cam = rgbCam; }
        return static_cast<int>(static_cast<CpuComputeBackend*>(b)->DemosaicBayer(cfa, w, h, black, camMul, cam, filters, out));
    }

    // Kernels::SeamBlend::BlendChunkContributors (SeamBlend.cpp:549-587).
    void ref_blend_chunk(const uint16_t** bufs, int k, int w, int h, uint16_t* out)
    {
        std::vector<const unsigned short*> v(bufs, bufs + k);
        std::vector<unsigned short> res;
        SB::BlendChunkContributors(v, w, h, res);
        std::memcpy(out, res.data(), res.size() * sizeof(uint16_t));
    }

    // The same chain with an explicit band count (6 for the full-size render).
    void ref_blend_chunk_bands(const uint16_t** bufs, int k, int w, int h, int bands, uint16_t* out)
    {
        std::vector<const unsigned short*> v(bufs, bufs + k);
        std::vector<unsigned short> res;
        BlendWithBands(v, w, h, bands, res);
        std::memcpy(out, res.data(), res.size() * sizeof(uint16_t));
    }

    // Detail::ComputeCoverageDistance (SeamBlend.cpp:206-242).
    void ref_coverage_distance(const uint8_t* cov, int w, int h, float* out)
    {
        std::vector<unsigned char> c(cov, cov + static_cast<size_t>(w) * h);
        std::vector<float> d;
        SB::Detail::ComputeCoverageDistance(c, w, h, d);
        std::memcpy(out, d.data(), d.size() * sizeof(float));
    }

    // Detail::ComputeOwnership (SeamBlend.cpp:244-261).
    void ref_ownership(const float** dists, int k, int w, int h, int32_t* owner)
    {
        size_t n = static_cast<size_t>(w) * h;
        std::vector<std::vector<float>> d(k);
        for (int i = 0; i < k; ++i) d[i].assign(dists[i], dists[i] + n);
        std::vector<int> o;
        SB::Detail::ComputeOwnership(d, w, h, o);
        for (size_t p = 0; p < n; ++p) owner[p] = o[p];
    }

    // Detail::ComputeCoverageBBox (SeamBlend.cpp:263-280); out = x0,y0,x1,y1.
    int ref_bbox(const uint8_t* cov, int w, int h, int32_t* out)
    {
        std::vector<unsigned char> c(cov, cov + static_cast<size_t>(w) * h);
        SB::Detail::BBox b = SB::Detail::ComputeCoverageBBox(c, w, h);
        out[0] = b.x0; out[1] = b.y0; out[2] = b.x1; out[3] = b.y1;
        return b.valid ? 1 : 0;
    }

    // Detail::RefineSeamDP (SeamBlend.cpp:293-445), owner updated in place.
    // Bounding boxes are derived from the distance fields the same way
    // BlendChunkContributors derives them from coverage.
    void ref_refine_seam(const uint16_t* imgI, const uint16_t* imgJ, const float* distI, const float* distJ,
                         int w, int h, int ci, int cj, int32_t* owner)
    {
        size_t n = static_cast<size_t>(w) * h;
        std::vector<float> dI(distI, distI + n), dJ(distJ, distJ + n);
        std::vector<unsigned char> cI(n), cJ(n);
        for (size_t p = 0; p < n; ++p) { cI[p] = dI[p] > 0.0f; cJ[p] = dJ[p] > 0.0f; }
        SB::Detail::BBox bI = SB::Detail::ComputeCoverageBBox(cI, w, h);
        SB::Detail::BBox bJ = SB::Detail::ComputeCoverageBBox(cJ, w, h);
        SB::Detail::BBox ov;
        std::vector<int> o(owner, owner + n);
        if (SB::Detail::IntersectBBox(bI, bJ, ov))
            SB::Detail::RefineSeamDP(imgI, imgJ, dI, dJ, w, h, ci, cj, bI, bJ, ov, o);
        for (size_t p = 0; p < n; ++p) owner[p] = o[p];
    }

    // Detail::MultiBandCompose (SeamBlend.cpp:447-546).
    void ref_compose(const uint16_t** bufs, const float** dists, const int32_t* owner, int k, int w, int h,
                     int bands, uint16_t* out)
    {
        size_t n = static_cast<size_t>(w) * h;
        std::vector<const unsigned short*> v(bufs, bufs + k);
        std::vector<std::vector<float>> d(k);
        for (int i = 0; i < k; ++i) d[i].assign(dists[i], dists[i] + n);
        std::vector<int> o(owner, owner + n);
        std::vector<unsigned short> res;
        SB::Detail::MultiBandCompose(v, d, o, w, h, bands, res);
        std::memcpy(out, res.data(), res.size() * sizeof(uint16_t));
    }

    // CPU-backend render of a list of output tiles, each treated as one
    // RenderExecutor chunk: per contributor WarpPerspective (dst->src matrix)
    // then ApplyGain when |gain-1| > 1e-6, then the seam blend with `bands`
    // levels.  Tasks are pulled by `threads` workers (the reference runs
    // hardware_concurrency()-1 of them).  Frames are host RGB48.  Tile i has
    // contributors contrib[contribOffset[i] .. contribOffset[i+1]).
    // Returns wall seconds; outputs go to out[i] (w*h*3 each) when non-null.
    double ref_render_tiles(int threads, int tier,
                            const uint16_t** frames, const int32_t* frameW, const int32_t* frameH,
                            const float* invH /* 9 per frame */, const float* gains,
                            int nTiles, const int32_t* tileRect /* x,y,w,h per tile */,
                            const int32_t* contribOffset, const int32_t* contrib,
                            int bands, uint16_t** out)
    {
        std::atomic<int> next{0};
        auto t0 = std::chrono::steady_clock::now();
        auto worker = [&]() {
            std::vector<std::vector<unsigned short>> warped;
            std::vector<unsigned short> res;
            for (;;)
            {
                int t = next.fetch_add(1);
                if (t >= nTiles) break;
                int tx = tileRect[4 * t], ty = tileRect[4 * t + 1], tw = tileRect[4 * t + 2], th = tileRect[4 * t + 3];
                size_t n3 = static_cast<size_t>(tw) * th * 3;
                int kBeg = contribOffset[t], kEnd = contribOffset[t + 1];
                warped.assign(kEnd - kBeg, std::vector<unsigned short>());
                std::vector<const unsigned short*> ptrs;
                for (int k = kBeg; k < kEnd; ++k)
                {
                    int f = contrib[k];
                    auto& wb = warped[k - kBeg];
                    wb.assign(n3, 0);
                    ref_warp(tier, frames[f], frameW[f], frameH[f], wb.data(), tw, th, invH + 9 * f, tx, ty);
                    if (std::fabs(gains[f] - 1.0f) > 1e-6f) ApplyGainCpu(wb.data(), static_cast<int>(n3), gains[f]);
                    ptrs.push_back(wb.data());
                }
                BlendWithBands(ptrs, tw, th, bands, res);
                if (out && out[t]) std::memcpy(out[t], res.data(), n3 * sizeof(uint16_t));
            }
        };
        std::vector<std::thread> pool;
        int nt = threads < 1 ? 1 : threads;
        for (int i = 0; i < nt; ++i) pool.emplace_back(worker);
        for (auto& th : pool) th.join();
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    // CPU-backend demosaic of a batch of CFA frames (RawIngestExecutor.cpp:90-93),
    // one frame per task on `threads` workers.  Returns wall seconds.
    double ref_demosaic_frames(int threads, int tier, int nFrames, const uint16_t** cfa, int w, int h,
                               uint16_t black, const float* camMul, const float* rgbCamFlat, uint32_t filters,
                               uint16_t** out)
    {
        std::atomic<int> next{0};
        auto t0 = std::chrono::steady_clock::now();
        auto worker = [&]() {
            for (;;)
            {
                int f = next.fetch_add(1);
                if (f >= nFrames) break;
                ref_demosaic(tier, cfa[f], w, h, black, camMul, rgbCamFlat, filters, out[f]);
            }
        };
        std::vector<std::thread> pool;
        int nt = threads < 1 ? 1 : threads;
        for (int i = 0; i < nt; ++i) pool.emplace_back(worker);
        for (auto& th : pool) th.join();
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
}

extern "C"
{
    // Inputs of the median cross-tier check in tests/engine_smoke/main.cpp:176-193:
    // 21 planes of 17x13x3 drawn from std::mt19937(777) with
    // uniform_int_distribution<int>(0, 4000) in plane order, then value 60000 at
    // index 100 of planes 0..2.  Written to out[21 * 663].
    void ref_engine_smoke_median_inputs(uint16_t* out)
    {
        const size_t plane = 17 * 13 * 3;
        std::mt19937 rng(777);
        std::uniform_int_distribution<int> dist(0, 4000);
        for (int i = 0; i < 21; ++i)
            for (size_t k = 0; k < plane; ++k) out[i * plane + k] = static_cast<uint16_t>(dist(rng));
        for (int i = 0; i < 3; ++i) out[i * plane + 100] = 60000;
    }
}
