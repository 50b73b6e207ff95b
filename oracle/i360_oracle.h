/*
 * Test infrastructure only (the oracle).  A plain-C restatement of the
 * reference's CPU render path (thnak/Image360, WindowsApp.Core), used by the
 * tests, the golden-fixture script and bench.py's CPU-baseline leg as the
 * checker.  The product never links or calls it.
 *
 * Pixel format everywhere: RGB48 = interleaved uint16 x3, row-major.  Every
 * function states the reference file:line it follows; the arithmetic is in the
 * same FP32 operation order (built with -ffp-contract=off, no FMA) so results
 * are bit-identical to the reference's scalar tier.
 */
#ifndef I360_ORACLE_H
#define I360_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* BayerDemosaic_Scalar.cpp:9-50 with BayerDemosaicKernels.h:10-75. */
void or_demosaic(const uint16_t* cfa, int w, int h, uint16_t black, const float* camMul4,
                 const float* rgbCam12, uint32_t filters, uint16_t* rgbOut);

/* WarpPerspective_Scalar.cpp:8-45 with WarpPerspectiveKernels.h:16-43.
 * invH maps destination -> source, row-major. */
void or_warp(const uint16_t* src, int sw, int sh, uint16_t* dst, int dw, int dh,
             const float* invH, int offX, int offY);

/* MedianStack_Scalar.cpp:8-24 with MedianStackKernels.h:19-55. */
void or_median(const uint16_t* const* inputs, int n, uint16_t* out, int w, int h, float sigma);

/* GainColorOps.cpp:16-26 (in place). */
void or_gain(uint16_t* data, int n, float gain);

/* GainColorOps.cpp:103-130: mean and standard deviation of CIE L, a, b over an
 * RGB48 image (per-pixel conversion GainColorOps.cpp:56-73). */
void or_lab_stats(const uint16_t* rgb, int w, int h, double* mean3, double* std3);

/* GainColorOps.cpp:132-156 (in place; back conversion GainColorOps.cpp:75-100). */
void or_reinhard(uint16_t* rgb, int w, int h, const double* srcMean, const double* srcStd,
                 const double* refMean, const double* refStd);

/* OverlapCulling.cpp:36-71 (ImageOverlapsChunk): 1 when the box of the
 * frame's projected corners overlaps the chunk.  f64: the FP64 form. */
int or_image_overlaps_chunk(const float* h9, int imageW, int imageH, int chunkX, int chunkY, int chunkW,
                            int chunkH);
int or_image_overlaps_chunk_f64(const float* h9, int imageW, int imageH, int chunkX, int chunkY, int chunkW,
                                int chunkH);

/* PanoramaExporter.cpp:9-24. */
float or_export_scale(int totalW, int totalH, int maxDimension);
void or_chunk_placement(int x, int y, int w, int h, float scale, int* out4);

/* The preview composite of PanoramaExporter.cpp:46-102: every chunk's RGB48
 * output (tiles[c], the chunk rectangle rects[4c..4c+3]; null = no render
 * output) placed in chunk order into an RGB8 canvas of the exported size,
 * nearest source pixel, 16 -> 8 bits by >> 8.  Writes the size to
 * outW/outH; returns 0 when the composite needs more than `capacity` bytes
 * or the arguments are invalid. */
int or_export_preview(const uint16_t* const* tiles, const int32_t* rects, int numTiles, int totalW, int totalH,
                      int maxDimension, uint8_t* out, long long capacity, int* outW, int* outH);

/* StorageEngine.cpp:130-144: int32 width, int32 height, the RGB48 samples. */
void or_frame_pixel_buffer(const uint16_t* data, int w, int h, uint8_t* out);

/* Tiff16Writer.cpp:40-97 as bytes (size or_tiff16_size(w, h)). */
long long or_tiff16_size(int w, int h);
void or_tiff16_bytes(const uint16_t* data, int w, int h, uint8_t* out);

/* HomographyMath.cpp:94-116.  Returns 1 on success, 0 when singular. */
int or_invert_h(const float* h, float* out);

/* SeamBlend.cpp:564-565: covered = any channel != 0. */
void or_coverage(const uint16_t* img, int w, int h, uint8_t* cov);

/* SeamBlend.cpp:206-242. */
void or_coverage_distance(const uint8_t* cov, int w, int h, float* dist);

/* SeamBlend.cpp:244-261. */
void or_ownership(const float* const* dists, int k, int w, int h, int32_t* owner);

/* SeamBlend.cpp:263-280; box = x0,y0,x1,y1; returns valid. */
int or_bbox(const uint8_t* cov, int w, int h, int32_t* box);

/* SeamBlend.cpp:293-445 for one (i, j) pair, owner updated in place. */
void or_refine_seam(const uint16_t* imgI, const uint16_t* imgJ, const float* distI, const float* distJ,
                    int w, int h, int ci, int cj, const int32_t* boxI, const int32_t* boxJ,
                    const int32_t* overlap, int32_t* owner);

/* SeamBlend.cpp:447-546. */
void or_compose(const uint16_t* const* bufs, const float* const* dists, const int32_t* owner, int k,
                int w, int h, int bands, uint16_t* out);

/* SeamBlend.cpp:549-587 with an explicit band count (5 = kDefaultNumBands). */
void or_blend_chunk(const uint16_t* const* bufs, int k, int w, int h, int bands, uint16_t* out);

/* Same chain, also returning the final owner map (after seam refinement). */
void or_blend_chunk_ex(const uint16_t* const* bufs, int k, int w, int h, int bands, uint16_t* out,
                       int32_t* ownerOut);

/* Band-count clamp of SeamBlend.cpp:457-459. */
int or_clamp_bands(int w, int h, int bands);

/* FP64 restatements for error reporting: the same steps with every FP32
 * operation done in double, quantised at the same points as the reference
 * (truncation at stage boundaries, +0.5 rounding at the blend output). */
void or_demosaic_f64(const uint16_t* cfa, int w, int h, uint16_t black, const float* camMul4,
                     const float* rgbCam12, uint32_t filters, uint16_t* rgbOut);
void or_warp_f64(const uint16_t* src, int sw, int sh, uint16_t* dst, int dw, int dh,
                 const double* invH, int offX, int offY);
void or_compose_f64(const uint16_t* const* bufs, const int32_t* owner, int k, int w, int h, int bands,
                    uint16_t* out);
void or_lab_stats_f64(const uint16_t* rgb, int w, int h, double* mean3, double* std3);
void or_reinhard_f64(uint16_t* rgb, int w, int h, const double* srcMean, const double* srcStd,
                     const double* refMean, const double* refStd);

/* Render a list of output tiles the way RenderExecutor::Execute does per chunk
 * (RenderExecutor.cpp:70-140): warp each contributor with its dst->src matrix,
 * ApplyGain when |gain-1| > 1e-6, then blend with `bands` levels.  `threads`
 * pthreads pull tiles from a shared counter.  Returns wall seconds. */
double or_render_tiles(int threads, const uint16_t* const* frames, const int32_t* frameW,
                       const int32_t* frameH, const float* invH, const float* gains, int nTiles,
                       const int32_t* tileRect, const int32_t* contribOffset, const int32_t* contrib,
                       int bands, uint16_t** out);

#ifdef __cplusplus
}
#endif

#endif
